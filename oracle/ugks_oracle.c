/*
 * ugks_oracle.c -- TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline; see the header).
 *
 * Plain-C restatement of the reference's second-order UGKS hot path for the planar Couette
 * case (x-periodic, diffuse moving walls at y=0 and y=H, FluxWall_type=1 + CouetteUseW2BWall,
 * UnifiedPhysicalOperators=.true., power-law viscosity).  Loop and summation order follow the
 * Fortran so that the restatement reproduces the reference's printed numbers to their digits.
 * File:line citations are relative to the reference project root.
 */
#include "ugks_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

#define PI_D 3.14159265358979323846264338327950288
static const double SMV = (double)FLT_MIN;   /* mod_Globaldata.f90:26 SMV = tiny(0.0_real32) */

struct uo_ctx {
    uo_params p;
    int nc;                       /* nx*ny */
    double area;
    double *u, *v, *w;
    double umax, vmax;
    double *h, *b, *W;
    double *sh, *sb;              /* [c][2][nvel] Van-Leer slopes; dir 0 = x, 1 = y */
    double *fxh, *fxb, *fxw;      /* x faces [j][i][..], face i between cells i-1 and i (periodic) */
    double *fyLh, *fyLb, *fyLw;   /* y faces [jf][i][..], jf = 0..ny; L flux */
    double *fyRh, *fyRb, *fyRw;   /* R flux (equal to L for interior faces) */
    double *res_w, *res_h, *res_b;  /* res_macro_flux_store, res_h/b_flux_store */
    double *rate_w, *stream_h, *stream_b;
    double *peq_h, *peq_b, *pcol_h, *pcol_b;
    double *wall_aero;            /* [2][nx][3] */
    double *cell_diag;            /* [nc][13] per-cell residual-norm terms, summed in cell order */
    int *cell_err;                /* [nc] per-cell status */
    /* ImplicitSteady state (mod_ImplicitState.f90) */
    double *dw, *dw_ghost;        /* delta_w [nc][4] and its halo snapshot from the last exchange */
    double *wt, *tau_t;           /* w_tilde [nc][4], tau_tilde [nc] */
    double *eq_h, *eq_b;          /* predicted equilibrium [nc][nvel] */
    double *dh, *db;              /* delta_h, delta_b [nc][nvel] */
    double *dh_ghost, *db_ghost;  /* halo snapshot of delta_h, delta_b */
    double *save_h, *save_b, *save_W;
    double ref_h, ref_b;          /* first-evaluation micro residual references */
    int ref_init;
    double m0;                    /* closed_mass_target (persistent M0) */
    double mass_scale;
    int streak;
    double dt;
    /* high-order S2 path (ugks_oracle_s2.c) */
    double *s2_rec;               /* reconstruction cache [nc][nvel][72] */
    double *s2_mh, *s2_mb, *s2_kxh, *s2_kxb, *s2_kyh, *s2_kyb;   /* volume targets [nc][nvel] */
    double *s2_kappa;             /* [nc][2x2] */
    double *lco_h, *lco_b;        /* low_collision_old [nc][nvel] */
    double *s2_facc;              /* per-cell face flux accumulators */
    void *s2_scr;                 /* per-thread closure scratch */
    /* S2CN2 explicit high-order step (ugks_oracle_s2.c) */
    int s2_ready;                 /* s2_mh.. hold the targets of the accepted state */
    double *cn_mh, *cn_mb, *cn_kxh, *cn_kxb, *cn_kyh, *cn_kyb, *cn_kappa;   /* targets of the proposal */
    double *cn_wn, *cn_hs, *cn_bs;   /* stream state W + res, h + res_h, b + res_b */
    double *cn_hn, *cn_bn;        /* proposal after the CN collision */
    double *cn_cell;              /* [nc][UO_CN_CELL] per-cell advance diagnostics */
    double cn_total0[4], cn_balance[4];   /* conservation ledger: initial totals, cumulative wall balance */
    /* research wall variants (ugks_oracle_s2.c) */
    double *s2_coef;              /* [nc][3 faces as s2_facc][f0 h, f0 b, k h, k b][nvel] leading / time coefficients */
    double *s2_facc0;             /* the accepted state's face accumulators while a predictor runs */
    double *v_inst;               /* [nc][3 faces][h nv, b nv] instantaneous fluxes at the predicted state */
    /* scratch: 24 work vectors per OpenMP thread */
    int nthr;
    double **tt;
};

#define NSCR 24
#define UO_CN_CELL 8
#define MAX_THREADS 256
static int g_threads = 1;   /* threads used by par_for; set by uo_set_threads */

static int host_cores(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n < 1 ? 1 : (n > MAX_THREADS ? MAX_THREADS : (int)n);
}

int uo_set_threads(int n) {
    g_threads = n > 0 ? (n > MAX_THREADS ? MAX_THREADS : n) : host_cores();
    return g_threads;
}

/* Minimal parallel-for over independent items: each worker takes item indices from an atomic
 * counter and passes its worker id (for per-thread scratch) to the body. */
typedef void (*par_body)(void* arg, int item, int tid);
typedef struct { par_body body; void* arg; int n, tid; atomic_int* next; } par_job;

static void* par_worker(void* vp) {
    par_job* j = (par_job*)vp;
    for (;;) {
        int i = atomic_fetch_add(j->next, 1);
        if (i >= j->n) break;
        j->body(j->arg, i, j->tid);
    }
    return NULL;
}

static void par_for(int n, par_body body, void* arg, int nthr) {
    if (nthr <= 1 || n <= 1) {
        for (int i = 0; i < n; ++i) body(arg, i, 0);
        return;
    }
    if (nthr > n) nthr = n;
    atomic_int next = 0;
    pthread_t th[MAX_THREADS];
    par_job jobs[MAX_THREADS];
    for (int t = 0; t < nthr; ++t) { jobs[t].body = body; jobs[t].arg = arg; jobs[t].n = n; jobs[t].tid = t; jobs[t].next = &next; }
    for (int t = 1; t < nthr; ++t) pthread_create(&th[t], NULL, par_worker, &jobs[t]);
    par_worker(&jobs[0]);
    for (int t = 1; t < nthr; ++t) pthread_join(th[t], NULL);
}

static double** scratch_t(uo_ctx* c, int tid) { return c->tt + (size_t)tid * NSCR; }

/* ------------------------------------------------------------------ kinetic math library */

/* GetPrimary (mod_Tools.f90:209-235) */
static int get_primary(const uo_params* p, const double w[4], double prim[4]) {
    for (int m = 0; m < 4; ++m) if (!isfinite(w[m])) return 101;
    if (w[0] <= 0.0) return 102;
    double denom = w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0];
    if (!isfinite(denom) || denom <= 0.0) return 103;
    prim[0] = w[0];
    prim[1] = w[1] / w[0];
    prim[2] = w[2] / w[0];
    prim[3] = 0.5 * w[0] / ((p->gamma - 1.0) * denom);
    return 0;
}

/* GetConserved (mod_Tools.f90:190-200) */
static void get_conserved(const uo_params* p, const double prim[4], double w[4]) {
    w[0] = prim[0];
    w[1] = prim[0] * prim[1];
    w[2] = prim[0] * prim[2];
    w[3] = 0.5 * prim[0] / (prim[3] * (p->gamma - 1.0)) + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]);
}

/* GetTau, power law (mod_Tools.f90:267-299) */
static int get_tau(const uo_params* p, const double prim[4], double* tau) {
    if (prim[0] <= 0.0 || prim[3] <= 0.0 || !isfinite(prim[0]) || !isfinite(prim[1]) ||
        !isfinite(prim[2]) || !isfinite(prim[3])) return 104;
    double mu = p->mu_ref * pow(1.0 / prim[3], p->omega);
    if (!isfinite(mu) || mu <= 0.0) return 105;
    *tau = mu / (0.5 * prim[0] / prim[3]);
    if (!isfinite(*tau) || *tau <= 0.0) return 106;
    return 0;
}

/* DiscreteMaxwell_LocalVec (mod_Tools.f90:44-64) */
static void maxwell(const uo_params* p, int n, const double* vn, const double* vt, const double prim[4],
                    double* H, double* B) {
    double pref = prim[0] * (prim[3] / PI_D);
    double bf = (double)p->ck / (2.0 * prim[3]);
    for (int k = 0; k < n; ++k) {
        double dvn = vn[k] - prim[1], dvt = vt[k] - prim[2];
        double v2 = dvn * dvn + dvt * dvt;
        double hk = pref * exp(-prim[3] * v2);
        H[k] = hk;
        B[k] = hk * bf;
    }
}

/* ShakhovPart_LocalVec, ck>0 branch (mod_Tools.f90:110-128) */
static void shakhov(const uo_params* p, int n, const double* H, const double* B, const double* vn,
                    const double* vt, const double qf[2], const double prim[4], double* Hp, double* Bp) {
    double coeff = 0.8 * (1.0 - p->pr) * prim[3] * prim[3] / prim[0];
    for (int k = 0; k < n; ++k) {
        double dvn = vn[k] - prim[1], dvt = vt[k] - prim[2];
        double v2 = dvn * dvn + dvt * dvt;
        double qdot = dvn * qf[0] + dvt * qf[1];
        double shH = 2.0 * prim[3] * v2 - 4.0;
        double shB = shH + 2.0 / (double)p->ck;
        Hp[k] = coeff * qdot * shH * H[k];
        Bp[k] = coeff * qdot * shB * B[k];
    }
}

/* GetHeatFlux_LocalVec (mod_Tools.f90:379-400) */
static void heat_flux(int n, const double* h, const double* b, const double* vn, const double* vt,
                      const double* wv, const double prim[4], double q[2]) {
    q[0] = 0.0; q[1] = 0.0;
    for (int k = 0; k < n; ++k) {
        double dvn = vn[k] - prim[1], dvt = vt[k] - prim[2];
        double v2 = dvn * dvn + dvt * dvt;
        q[0] = q[0] + 0.5 * wv[k] * dvn * (v2 * h[k] + b[k]);
        q[1] = q[1] + 0.5 * wv[k] * dvt * (v2 * h[k] + b[k]);
    }
}

/* MomentConserved (mod_ImplicitCommon.f90:32-40): Fortran sum() intrinsic, sequential */
static void moment_conserved(int n, const double* h, const double* b, const double* u, const double* v,
                             const double* wl, double m[4]) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int k = 0; k < n; ++k) {
        s0 += wl[k] * h[k];
        s1 += wl[k] * u[k] * h[k];
        s2 += wl[k] * v[k] * h[k];
        s3 += wl[k] * ((u[k] * u[k] + v[k] * v[k]) * h[k] + b[k]);
    }
    m[0] = s0; m[1] = s1; m[2] = s2; m[3] = 0.5 * s3;
}

/* SolveDense4 (mod_ImplicitCommon.f90:84-113): Gauss-Jordan with partial pivoting.
 * m is row-major m[r*4+c]. */
int uo_solve_dense4(const double m[16], const double rhs[4], double sol[4]) {
    double a[4][5];
    double pscale = 0.0;
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) { a[r][c] = m[r * 4 + c]; if (fabs(m[r * 4 + c]) > pscale) pscale = fabs(m[r * 4 + c]); }
        a[r][4] = rhs[r];
    }
    if (pscale < DBL_MIN) pscale = DBL_MIN;
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r) if (fabs(a[r][col]) > fabs(a[piv][col])) piv = r;
        if (fabs(a[piv][col]) <= 1000.0 * DBL_EPSILON * pscale) return 0;
        if (piv != col) for (int c = 0; c < 5; ++c) { double t = a[col][c]; a[col][c] = a[piv][c]; a[piv][c] = t; }
        double d = a[col][col];
        for (int c = 0; c < 5; ++c) a[col][c] = a[col][c] / d;
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            double f = a[r][col];
            for (int c = 0; c < 5; ++c) a[r][c] = a[r][c] - f * a[col][c];
        }
    }
    for (int r = 0; r < 4; ++r) { sol[r] = a[r][4]; if (!isfinite(sol[r])) return 0; }
    return 1;
}

/* ProjectToConservedMoments (mod_ImplicitCommon.f90:42-82).  Returns 1 when ok. */
int uo_project_moments(int n, double* h, double* b, const double target[4], const double* u,
                       const double* v, const double* wl, const double* ref_h, const double* ref_b) {
    for (int m = 0; m < 4; ++m) if (!isfinite(target[m])) return 0;
    for (int k = 0; k < n; ++k) if (!isfinite(h[k]) || !isfinite(b[k])) return 0;
    double mom[4], rhs[4], gram[16] = {0}, lam[4];
    moment_conserved(n, h, b, u, v, wl, mom);
    for (int m = 0; m < 4; ++m) rhs[m] = target[m] - mom[m];
    double sh = 0.0, sb = 0.0;
    for (int k = 0; k < n; ++k) { if (fabs(ref_h[k]) > sh) sh = fabs(ref_h[k]); if (fabs(ref_b[k]) > sb) sb = fabs(ref_b[k]); }
    if (sh < 1.0) sh = 1.0;
    if (sb < 1.0) sb = 1.0;
    const double kb[4] = {0.0, 0.0, 0.0, 0.5};
    for (int k = 0; k < n; ++k) {
        double kh[4] = {1.0, u[k], v[k], 0.5 * (u[k] * u[k] + v[k] * v[k])};
        double wh = fmax(fabs(ref_h[k]), DBL_EPSILON * sh);
        double wb = fmax(fabs(ref_b[k]), DBL_EPSILON * sb);
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 4; ++c)
                gram[a * 4 + c] = gram[a * 4 + c] + wl[k] * (wh * kh[a] * kh[c] + wb * kb[a] * kb[c]);
    }
    if (!uo_solve_dense4(gram, rhs, lam)) return 0;
    for (int k = 0; k < n; ++k) {
        double kh[4] = {1.0, u[k], v[k], 0.5 * (u[k] * u[k] + v[k] * v[k])};
        double wh = fmax(fabs(ref_h[k]), DBL_EPSILON * sh);
        double wb = fmax(fabs(ref_b[k]), DBL_EPSILON * sb);
        h[k] = h[k] + wh * (kh[0] * lam[0] + kh[1] * lam[1] + kh[2] * lam[2] + kh[3] * lam[3]);
        b[k] = b[k] + 0.5 * wb * lam[3];
    }
    moment_conserved(n, h, b, u, v, wl, mom);
    double rs = 1.0;
    for (int m = 0; m < 4; ++m) if (fabs(target[m]) > rs) rs = fabs(target[m]);
    double err = 0.0;
    for (int m = 0; m < 4; ++m) if (fabs(mom[m] - target[m]) > err) err = fabs(mom[m] - target[m]);
    for (int k = 0; k < n; ++k) if (!isfinite(h[k]) || !isfinite(b[k])) return 0;
    return err <= 1.0e-10 * rs;
}

/* MicroSlope (mod_Evolution.f90:1792-1800) */
static void micro_slope(int ck, const double prim[4], const double sw[4], double a[4]) {
    double r = prim[0], U = prim[1], V = prim[2], L = prim[3];
    a[3] = 4.0 * (L * L) / ((double)(ck + 2) * r) *
           (2.0 * sw[3] - 2.0 * U * sw[1] - 2.0 * V * sw[2] + sw[0] * (U * U + V * V - 0.5 * (double)(ck + 2) / L));
    a[2] = 2.0 * L / r * (sw[2] - V * sw[0]) - V * a[3];
    a[1] = 2.0 * L / r * (sw[1] - U * sw[0]) - U * a[3];
    a[0] = sw[0] / r - U * a[1] - V * a[2] - 0.5 * (U * U + V * V + 0.5 * (double)(ck + 2) / L) * a[3];
}

#define MNUM 6
#define MTUM 5
/* CalcMoment (mod_Evolution.f90:1810-1842) */
static void calc_moment(int ck, const double prim[4], double Mu[MNUM + 1], double Mv[MTUM + 1], double Mxi[3],
                        double MuL[MNUM + 1], double MuR[MNUM + 1]) {
    double U = prim[1], L = prim[3];
    MuL[0] = 0.5 * erfc(-sqrt(L) * U);
    MuL[1] = U * MuL[0] + 0.5 * exp(-L * U * U) / sqrt(PI_D * L);
    MuR[0] = 0.5 * erfc(sqrt(L) * U);
    MuR[1] = U * MuR[0] - 0.5 * exp(-L * U * U) / sqrt(PI_D * L);
    for (int i = 2; i <= MNUM; ++i) {
        MuL[i] = U * MuL[i - 1] + 0.5 * (double)(i - 1) * MuL[i - 2] / L;
        MuR[i] = U * MuR[i - 1] + 0.5 * (double)(i - 1) * MuR[i - 2] / L;
    }
    for (int i = 0; i <= MNUM; ++i) Mu[i] = MuL[i] + MuR[i];
    Mv[0] = 1.0;
    Mv[1] = prim[2];
    for (int i = 2; i <= MTUM; ++i) Mv[i] = prim[2] * Mv[i - 1] + 0.5 * (double)(i - 1) * Mv[i - 2] / L;
    Mxi[0] = 1.0;
    Mxi[1] = 0.5 * (double)ck / L;
    Mxi[2] = (double)ck * ((double)ck + 2.0) / (4.0 * L * L);
}

/* Moment_uvxi (mod_Evolution.f90:1853-1862) */
static void moment_uvxi(const double* Mu, const double* Mv, const double* Mxi, int al, int be, int de, double o[4]) {
    o[0] = Mu[al] * Mv[be] * Mxi[de / 2];
    o[1] = Mu[al + 1] * Mv[be] * Mxi[de / 2];
    o[2] = Mu[al] * Mv[be + 1] * Mxi[de / 2];
    o[3] = 0.5 * (Mu[al + 2] * Mv[be] * Mxi[de / 2] + Mu[al] * Mv[be + 2] * Mxi[de / 2] + Mu[al] * Mv[be] * Mxi[(de + 2) / 2]);
}

/* Moment_auvxi (mod_Evolution.f90:1874-1885) */
static void moment_auvxi(const double a[4], const double* Mu, const double* Mv, const double* Mxi, int al, int be,
                         double o[4]) {
    double t0[4], t1[4], t2[4], t3[4], t4[4], t5[4];
    moment_uvxi(Mu, Mv, Mxi, al + 0, be + 0, 0, t0);
    moment_uvxi(Mu, Mv, Mxi, al + 1, be + 0, 0, t1);
    moment_uvxi(Mu, Mv, Mxi, al + 0, be + 1, 0, t2);
    moment_uvxi(Mu, Mv, Mxi, al + 2, be + 0, 0, t3);
    moment_uvxi(Mu, Mv, Mxi, al + 0, be + 2, 0, t4);
    moment_uvxi(Mu, Mv, Mxi, al + 0, be + 0, 2, t5);
    for (int m = 0; m < 4; ++m)
        o[m] = a[0] * t0[m] + a[1] * t1[m] + a[2] * t2[m] + 0.5 * a[3] * t3[m] + 0.5 * a[3] * t4[m] + 0.5 * a[3] * t5[m];
}

/* Mt(1..5) time-integration coefficients (mod_Evolution.f90:346-350) */
static void time_coeffs(double dt, double tau, double Mt[5]) {
    Mt[3] = tau * (1.0 - exp(-dt / tau));
    Mt[4] = -tau * dt * exp(-dt / tau) + tau * Mt[3];
    Mt[0] = dt - Mt[3];
    Mt[1] = -tau * Mt[0] + Mt[4];
    Mt[2] = 0.5 * (dt * dt) - tau * Mt[0];
}

/* PrepareNativeFaceEquilibrium (mod_Evolution.f90:16-30) */
static int face_equilibrium(const uo_params* p, int n, const double* vn, const double* vt, const double* wv,
                            const double prim[4], double* H, double* B, double* rh, double* rb) {
    maxwell(p, n, vn, vt, prim, H, B);
    memcpy(rh, H, sizeof(double) * n);
    memcpy(rb, B, sizeof(double) * n);
    double target[4];
    get_conserved(p, prim, target);
    return uo_project_moments(n, H, B, target, vn, vt, wv, rh, rb) ? 0 : 446;
}

/* ------------------------------------------------------------------ context */

uo_ctx* uo_create(const uo_params* p, const double* u, const double* v, const double* w) {
    uo_ctx* c = (uo_ctx*)calloc(1, sizeof(uo_ctx));
    c->p = *p;
    int nv = p->nvel, nx = p->nx, ny = p->ny;
    c->nc = nx * ny;
    c->area = fabs((-p->dx) * (-p->dy) - (p->dx) * (-p->dy)) * 0.5;  /* rectangle area, mod_InitializeFlow.f90:388-389 */
    c->u = (double*)malloc(sizeof(double) * nv);
    c->v = (double*)malloc(sizeof(double) * nv);
    c->w = (double*)malloc(sizeof(double) * nv);
    memcpy(c->u, u, sizeof(double) * nv);
    memcpy(c->v, v, sizeof(double) * nv);
    memcpy(c->w, w, sizeof(double) * nv);
    c->umax = -INFINITY; c->vmax = -INFINITY;
    for (int k = 0; k < nv; ++k) { if (u[k] > c->umax) c->umax = u[k]; if (v[k] > c->vmax) c->vmax = v[k]; }
    size_t S = (size_t)c->nc * nv;
    c->h = (double*)calloc(S, sizeof(double));
    c->b = (double*)calloc(S, sizeof(double));
    c->W = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->sh = (double*)calloc(2 * S, sizeof(double));
    c->sb = (double*)calloc(2 * S, sizeof(double));
    c->fxh = (double*)calloc(S, sizeof(double));
    c->fxb = (double*)calloc(S, sizeof(double));
    c->fxw = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    size_t SY = (size_t)(ny + 1) * nx * nv;
    c->fyLh = (double*)calloc(SY, sizeof(double));
    c->fyLb = (double*)calloc(SY, sizeof(double));
    c->fyRh = (double*)calloc(SY, sizeof(double));
    c->fyRb = (double*)calloc(SY, sizeof(double));
    c->fyLw = (double*)calloc((size_t)(ny + 1) * nx * 4, sizeof(double));
    c->fyRw = (double*)calloc((size_t)(ny + 1) * nx * 4, sizeof(double));
    c->res_w = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->res_h = (double*)calloc(S, sizeof(double));
    c->res_b = (double*)calloc(S, sizeof(double));
    c->rate_w = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->stream_h = (double*)calloc(S, sizeof(double));
    c->stream_b = (double*)calloc(S, sizeof(double));
    c->peq_h = (double*)calloc(S, sizeof(double));
    c->peq_b = (double*)calloc(S, sizeof(double));
    c->pcol_h = (double*)calloc(S, sizeof(double));
    c->pcol_b = (double*)calloc(S, sizeof(double));
    c->wall_aero = (double*)calloc((size_t)2 * nx * 3, sizeof(double));
    c->cell_diag = (double*)calloc((size_t)c->nc * 13, sizeof(double));
    c->cell_err = (int*)calloc((size_t)c->nc, sizeof(int));
    c->dw = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->dw_ghost = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->wt = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->tau_t = (double*)calloc((size_t)c->nc, sizeof(double));
    c->eq_h = (double*)calloc(S, sizeof(double));
    c->eq_b = (double*)calloc(S, sizeof(double));
    c->dh = (double*)calloc(S, sizeof(double));
    c->db = (double*)calloc(S, sizeof(double));
    c->dh_ghost = (double*)calloc(S, sizeof(double));
    c->db_ghost = (double*)calloc(S, sizeof(double));
    c->save_h = (double*)calloc(S, sizeof(double));
    c->save_b = (double*)calloc(S, sizeof(double));
    c->save_W = (double*)calloc((size_t)c->nc * 4, sizeof(double));
    c->mass_scale = 1.0;
    c->nthr = MAX_THREADS < host_cores() ? MAX_THREADS : host_cores();
    c->tt = (double**)calloc((size_t)c->nthr * NSCR, sizeof(double*));
    for (int i = 0; i < c->nthr * NSCR; ++i) c->tt[i] = (double*)calloc(nv, sizeof(double));
    return c;
}

static void s2_free(uo_ctx* c);
static void cn_free(uo_ctx* c);
void uo_destroy(uo_ctx* c) {
    if (!c) return;
    s2_free(c);
    cn_free(c);
    double* ptrs[] = {c->u, c->v, c->w, c->h, c->b, c->W, c->sh, c->sb, c->fxh, c->fxb, c->fxw, c->fyLh, c->fyLb,
                      c->fyRh, c->fyRb, c->fyLw, c->fyRw, c->res_w, c->res_h, c->res_b, c->rate_w, c->stream_h,
                      c->stream_b, c->peq_h, c->peq_b, c->pcol_h, c->pcol_b, c->wall_aero};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
    for (int i = 0; i < c->nthr * NSCR; ++i) free(c->tt[i]);
    free(c->tt);
    free(c->cell_diag);
    free(c->cell_err);
    double* extra[] = {c->dw, c->dw_ghost, c->wt, c->tau_t, c->eq_h, c->eq_b, c->dh, c->db, c->dh_ghost, c->db_ghost,
                       c->save_h, c->save_b, c->save_W};
    for (size_t i = 0; i < sizeof(extra) / sizeof(extra[0]); ++i) free(extra[i]);
    free(c);
}

void uo_set_state(uo_ctx* c, const double* h, const double* b, const double* W) {
    size_t S = (size_t)c->nc * c->p.nvel;
    memcpy(c->h, h, S * sizeof(double));
    memcpy(c->b, b, S * sizeof(double));
    memcpy(c->W, W, (size_t)c->nc * 4 * sizeof(double));
}

void uo_get_state(const uo_ctx* c, double* h, double* b, double* W) {
    size_t S = (size_t)c->nc * c->p.nvel;
    if (h) memcpy(h, c->h, S * sizeof(double));
    if (b) memcpy(b, c->b, S * sizeof(double));
    if (W) memcpy(W, c->W, (size_t)c->nc * 4 * sizeof(double));
}

const double* uo_res_macro(const uo_ctx* c) { return c->res_w; }
const double* uo_res_h(const uo_ctx* c) { return c->res_h; }
const double* uo_res_b(const uo_ctx* c) { return c->res_b; }
const double* uo_wall_aero(const uo_ctx* c) { return c->wall_aero; }
const double* uo_face_x_h(const uo_ctx* c) { return c->fxh; }
const double* uo_face_y_h(const uo_ctx* c) { return c->fyLh; }
const double* uo_face_x_w(const uo_ctx* c) { return c->fxw; }
const double* uo_face_y_w(const uo_ctx* c) { return c->fyLw; }
const double* uo_phys_eq_h(const uo_ctx* c) { return c->peq_h; }
const double* uo_phys_col_h(const uo_ctx* c) { return c->pcol_h; }
const double* uo_phys_col_b(const uo_ctx* c) { return c->pcol_b; }

/* InitFlow_Freestream (mod_InitializeFlow.f90:826-856) followed by the cold-start
 * EnforceAcceptedMomentCompatibility of InitializeSteadyImplicit (mod_SteadyImplicit.f90:28-42,
 * mod_ImplicitMicro.f90 EnforceAcceptedMomentCompatibility). */
int uo_init_freestream(uo_ctx* c, double rho, double U, double V, double tnative) {
    const uo_params* p = &c->p;
    int nv = p->nvel;
    double prim[4] = {rho, U, V, 1.0 / tnative}, W[4];
    get_conserved(p, prim, W);
    double** T = scratch_t(c, 0);
    double *H = T[0], *B = T[1], *rh = T[2], *rb = T[3];
    maxwell(p, nv, c->u, c->v, prim, H, B);
    for (int cell = 0; cell < c->nc; ++cell) {
        memcpy(c->h + (size_t)cell * nv, H, sizeof(double) * nv);
        memcpy(c->b + (size_t)cell * nv, B, sizeof(double) * nv);
        memcpy(c->W + cell * 4, W, sizeof(double) * 4);
    }
    for (int cell = 0; cell < c->nc; ++cell) {
        double* hc = c->h + (size_t)cell * nv;
        double* bc = c->b + (size_t)cell * nv;
        memcpy(rh, hc, sizeof(double) * nv);
        memcpy(rb, bc, sizeof(double) * nv);
        if (!uo_project_moments(nv, hc, bc, c->W + cell * 4, c->u, c->v, c->w, rh, rb)) return 447;
    }
    return 0;
}

/* TimeStep (mod_Solve.f90:373-421), Time_global_varying */
double uo_timestep(uo_ctx* c) {
    const uo_params* p = &c->p;
    double tmin = INFINITY;
    for (int cell = 0; cell < c->nc; ++cell) {
        double prim[4];
        if (get_primary(p, c->W + cell * 4, prim)) return NAN;
        double sos = sqrt(0.5 * p->gamma / prim[3]);
        double a = fmax(c->umax, fabs(prim[1]) + sos);
        double bq = fmax(c->vmax, fabs(prim[2]) + sos);
        double dtl = p->cfl * c->area / (p->dy * a + p->dx * bq);
        if (dtl < tmin) tmin = dtl;
    }
    return tmin;
}

/* ------------------------------------------------------------------ Interpolation */

/* Interp_VanLeer limiter (mod_Interpolation.f90:142-170) */
static inline double vanleer(double sL, double sR) {
    return (copysign(1.0, sR) + copysign(1.0, sL)) * fabs(sR) * fabs(sL) / (fabs(sR) + fabs(sL) + SMV);
}

/* Interpolation (mod_Interpolation.f90:26-90) on one domain: x-periodic Van Leer for every cell;
 * y Van Leer for rows 2..ny-1 and the one-sided InterpBoundary slope on the wall rows
 * (UnifiedPhysicalOperators skips the wall rows in the inner loop, :40-45,78-88). */
void uo_interpolation(uo_ctx* c) {
    const uo_params* p = &c->p;
    int nx = p->nx, ny = p->ny, nv = p->nvel;
    double dL = 0.5 * (p->dx + p->dx), dR = 0.5 * (p->dx + p->dx);
    double eL = 0.5 * (p->dy + p->dy);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int cc = j * nx + i, cl = j * nx + (i + nx - 1) % nx, cr = j * nx + (i + 1) % nx;
            double *sh = c->sh + ((size_t)cc * 2 + 0) * nv, *sb = c->sb + ((size_t)cc * 2 + 0) * nv;
            const double *h0 = c->h + (size_t)cc * nv, *hl = c->h + (size_t)cl * nv, *hr = c->h + (size_t)cr * nv;
            const double *b0 = c->b + (size_t)cc * nv, *bl = c->b + (size_t)cl * nv, *br = c->b + (size_t)cr * nv;
            for (int k = 0; k < nv; ++k) {
                sh[k] = vanleer((h0[k] - hl[k]) / dL, (hr[k] - h0[k]) / dR);
                sb[k] = vanleer((b0[k] - bl[k]) / dL, (br[k] - b0[k]) / dR);
            }
        }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int cc = j * nx + i;
            double *sh = c->sh + ((size_t)cc * 2 + 1) * nv, *sb = c->sb + ((size_t)cc * 2 + 1) * nv;
            if (j == 0 || j == ny - 1) {
                int lo = (j == 0) ? cc : (j - 1) * nx + i;
                int hi = (j == 0) ? (j + 1) * nx + i : cc;
                const double *hl = c->h + (size_t)lo * nv, *hr = c->h + (size_t)hi * nv;
                const double *bl = c->b + (size_t)lo * nv, *br = c->b + (size_t)hi * nv;
                for (int k = 0; k < nv; ++k) {
                    sh[k] = (hr[k] - hl[k]) / eL;
                    sb[k] = (br[k] - bl[k]) / eL;
                }
            } else {
                int cl = (j - 1) * nx + i, cr = (j + 1) * nx + i;
                const double *h0 = c->h + (size_t)cc * nv, *hl = c->h + (size_t)cl * nv, *hr = c->h + (size_t)cr * nv;
                const double *b0 = c->b + (size_t)cc * nv, *bl = c->b + (size_t)cl * nv, *br = c->b + (size_t)cr * nv;
                for (int k = 0; k < nv; ++k) {
                    sh[k] = vanleer((h0[k] - hl[k]) / eL, (hr[k] - h0[k]) / eL);
                    sb[k] = vanleer((b0[k] - bl[k]) / eL, (br[k] - b0[k]) / eL);
                }
            }
        }
}

/* ------------------------------------------------------------------ Evolution */

/* LocalFrame / GlobalFrame (mod_Tools.f90:150-183) */
static void local_frame(const double w[4], double cx, double cy, double o[4]) {
    o[0] = w[0]; o[1] = w[1] * cx + w[2] * cy; o[2] = -w[1] * cy + w[2] * cx; o[3] = w[3];
}
static void global_frame(const double w[4], double cx, double cy, double o[4]) {
    o[0] = w[0]; o[1] = w[1] * cx - w[2] * cy; o[2] = w[1] * cy + w[2] * cx; o[3] = w[3];
}

/* CalcFlux_MultiDimension (mod_Evolution.f90:186-492) for an interior face.
 * dir 0: vertical face (normal x, cosx=1, cosy=-0); dir 1: horizontal face (cosx=-0, cosy=1).
 * Output: micro flux Fh,Fb (already times face length) and macro flux Fw (MomentConserved of it). */
static int interior_face(uo_ctx* c, int tid, int dir, int cl, int cr, double dt, double* Fh, double* Fb,
                         double Fw[4]) {
    const uo_params* p = &c->p;
    int nv = p->nvel;
    double cx = dir == 0 ? 1.0 : -0.0, cy = dir == 0 ? -0.0 : 1.0;
    double flen = dir == 0 ? p->dy : p->dx;
    double len = dir == 0 ? p->dx : p->dy;   /* leftCell%length(idx) == rightCell%length(idx) */
    double** T = scratch_t(c, tid);
    double *vn = T[0], *vt = T[1], *dl = T[2], *hv = T[3], *bv = T[4], *shn = T[5], *sbn = T[6];
    double *sht = T[7], *sbt = T[8], *H0 = T[9], *B0 = T[10], *Hp = T[11], *Bp = T[12];
    double *rh = T[13], *rb = T[14];
    const double *hL = c->h + (size_t)cl * nv, *hR = c->h + (size_t)cr * nv;
    const double *bL = c->b + (size_t)cl * nv, *bR = c->b + (size_t)cr * nv;
    const double *shL = c->sh + (size_t)cl * 2 * nv, *shR = c->sh + (size_t)cr * 2 * nv;
    const double *sbL = c->sb + (size_t)cl * 2 * nv, *sbR = c->sb + (size_t)cr * 2 * nv;
    int nd = dir, td = 1 - dir;
    for (int k = 0; k < nv; ++k) {
        vn[k] = c->u[k] * cx + c->v[k] * cy;
        vt[k] = -c->u[k] * cy + c->v[k] * cx;
        dl[k] = (copysign(1.0, vn[k]) + 1.0) / 2.0;
    }
    for (int k = 0; k < nv; ++k) {
        double dL = dl[k], dR = 1.0 - dL;
        hv[k] = (hL[k] + 0.5 * len * shL[nd * nv + k]) * dL + (hR[k] - 0.5 * len * shR[nd * nv + k]) * dR;
        bv[k] = (bL[k] + 0.5 * len * sbL[nd * nv + k]) * dL + (bR[k] - 0.5 * len * sbR[nd * nv + k]) * dR;
        shn[k] = shL[nd * nv + k] * dL + shR[nd * nv + k] * dR;
        sbn[k] = sbL[nd * nv + k] * dL + sbR[nd * nv + k] * dR;
        if (dir == 0) {
            sht[k] = shL[td * nv + k] * dL + shR[td * nv + k] * dR;
            sbt[k] = sbL[td * nv + k] * dL + sbR[td * nv + k] * dR;
        } else {
            sht[k] = -(shL[td * nv + k] * dL + shR[td * nv + k] * dR);
            sbt[k] = -(sbL[td * nv + k] * dL + sbR[td * nv + k] * dR);
        }
    }
    double cv[4] = {0, 0, 0, 0};
    for (int k = 0; k < nv; ++k) {
        double wk = c->w[k], a = vn[k], t = vt[k], v2 = a * a + t * t;
        cv[0] = cv[0] + wk * hv[k];
        cv[1] = cv[1] + wk * a * hv[k];
        cv[2] = cv[2] + wk * t * hv[k];
        cv[3] = cv[3] + 0.5 * wk * (v2 * hv[k] + bv[k]);
    }
    double prim[4];
    int e = get_primary(p, cv, prim);
    if (e) return e;
    double wl[4], wr[4], sw[4], aL[4], aR[4], bs[4], aT[4];
    local_frame(c->W + cl * 4, cx, cy, wl);
    local_frame(c->W + cr * 4, cx, cy, wr);
    for (int m = 0; m < 4; ++m) sw[m] = (cv[m] - wl[m]) / (0.5 * len);
    micro_slope(p->ck, prim, sw, aL);
    for (int m = 0; m < 4; ++m) sw[m] = (wr[m] - cv[m]) / (0.5 * len);
    micro_slope(p->ck, prim, sw, aR);
    double swt[4] = {0, 0, 0, 0};
    for (int k = 0; k < nv; ++k) {
        double wk = c->w[k], a = vn[k], t = vt[k], v2 = a * a + t * t;
        swt[0] = swt[0] + wk * sht[k];
        swt[1] = swt[1] + wk * a * sht[k];
        swt[2] = swt[2] + wk * t * sht[k];
        swt[3] = swt[3] + 0.5 * wk * (v2 * sht[k] + sbt[k]);
    }
    micro_slope(p->ck, prim, swt, bs);
    double Mu[MNUM + 1], MuL[MNUM + 1], MuR[MNUM + 1], Mv[MTUM + 1], Mxi[3];
    calc_moment(p->ck, prim, Mu, Mv, Mxi, MuL, MuR);
    double MauL[4], MauR[4], Mbv[4];
    moment_auvxi(aL, MuL, Mv, Mxi, 1, 0, MauL);
    moment_auvxi(aR, MuR, Mv, Mxi, 1, 0, MauR);
    moment_auvxi(bs, Mu, Mv, Mxi, 0, 1, Mbv);
    for (int m = 0; m < 4; ++m) sw[m] = -prim[0] * (MauL[m] + MauR[m] + Mbv[m]);
    micro_slope(p->ck, prim, sw, aT);
    double tau;
    e = get_tau(p, prim, &tau);
    if (e) return e;
    double Mt[5];
    time_coeffs(dt, tau, Mt);
    /* the Maxwellian-part macro flux (mod_Evolution.f90:356-404) is overwritten by the
     * MomentConserved of the micro flux in unified mode (:470-473); only the micro flux matters. */
    e = face_equilibrium(p, nv, vn, vt, c->w, prim, H0, B0, rh, rb);
    if (e) return e;
    double qf[2];
    heat_flux(nv, hv, bv, vn, vt, c->w, prim, qf);
    shakhov(p, nv, H0, B0, vn, vt, qf, prim, Hp, Bp);
    for (int k = 0; k < nv; ++k) {
        double a = vn[k], t = vt[k], v2 = a * a + t * t;
        double dL = dl[k], dR = 1.0 - dL;
        double slh = a * shn[k] + t * sht[k];
        double slb = a * sbn[k] + t * sbt[k];
        double H = H0[k], B = B0[k];
        double h_aL = aL[0] * H + aL[1] * a * H + aL[2] * t * H + 0.5 * aL[3] * (v2 * H + B);
        double h_aR = aR[0] * H + aR[1] * a * H + aR[2] * t * H + 0.5 * aR[3] * (v2 * H + B);
        double h_b = bs[0] * H + bs[1] * a * H + bs[2] * t * H + 0.5 * bs[3] * (v2 * H + B);
        double h_aT = aT[0] * H + aT[1] * a * H + aT[2] * t * H + 0.5 * aT[3] * (v2 * H + B);
        double b_aL = aL[0] * B + aL[1] * a * B + aL[2] * t * B + 0.5 * aL[3] * (v2 * B + Mxi[2] * H);
        double b_aR = aR[0] * B + aR[1] * a * B + aR[2] * t * B + 0.5 * aR[3] * (v2 * B + Mxi[2] * H);
        double b_b = bs[0] * B + bs[1] * a * B + bs[2] * t * B + 0.5 * bs[3] * (v2 * B + Mxi[2] * H);
        double b_aT = aT[0] * B + aT[1] * a * B + aT[2] * t * B + 0.5 * aT[3] * (v2 * B + Mxi[2] * H);
        double fh = Mt[0] * a * (H + Hp[k]) + Mt[1] * a * a * (h_aL * dL + h_aR * dR) + Mt[1] * a * t * h_b +
                    Mt[2] * a * h_aT + Mt[3] * a * hv[k] - Mt[4] * a * slh;
        double fb = Mt[0] * a * (B + Bp[k]) + Mt[1] * a * a * (b_aL * dL + b_aR * dR) + Mt[1] * a * t * b_b +
                    Mt[2] * a * b_aT + Mt[3] * a * bv[k] - Mt[4] * a * slb;
        Fh[k] = flen * fh;
        Fb[k] = flen * fb;
    }
    moment_conserved(nv, Fh, Fb, c->u, c->v, c->w, Fw);
    return 0;
}

/* W2BMultiscaleFluxBoundary (mod_Evolution.f90:1888-2449) for the horizontal wall faces.
 * side = -1 (Lside, bottom wall, face below row 0) or +1 (Rside, top wall). */
static int wall_face(uo_ctx* c, int tid, int side, int cell, int iw, double dt, double* Fh, double* Fb, double Fw[4],
                     double aero[3]) {
    const uo_params* p = &c->p;
    int nv = p->nvel;
    double cx = -0.0, cy = 1.0, flen = p->dx, len = p->dy;
    double rot = -(double)side;
    double** T = scratch_t(c, tid);
    double *vn = T[0], *vt = T[1], *dl = T[2], *hv = T[3], *bv = T[4], *shn = T[5], *sbn = T[6];
    double *sht = T[7], *sbt = T[8], *Hg = T[9], *Bg = T[10], *Hp = T[11], *Bp = T[12];
    double *rh = T[13], *rb = T[14], *Hw = T[15], *Bw = T[16];
    const double *h = c->h + (size_t)cell * nv, *b = c->b + (size_t)cell * nv;
    const double *sh = c->sh + (size_t)cell * 2 * nv, *sb = c->sb + (size_t)cell * 2 * nv;
    for (int k = 0; k < nv; ++k) {
        vn[k] = c->u[k] * cx + c->v[k] * cy;
        vt[k] = -c->u[k] * cy + c->v[k] * cx;
        dl[k] = (copysign(1.0, vn[k]) * rot + 1.0) / 2.0;
    }
    for (int k = 0; k < nv; ++k) {
        shn[k] = sh[nv + k];
        sbn[k] = sb[nv + k];
        sht[k] = -sh[k];
        sbt[k] = -sb[k];
    }
    for (int k = 0; k < nv; ++k) {
        hv[k] = h[k] - rot * 0.5 * len * shn[k];
        bv[k] = b[k] - rot * 0.5 * len * sbn[k];
    }
    double bc[4] = {1.0, p->wall_ux[iw], 0.0, 1.0 / p->wall_tnative[iw]};
    double prim_w[4], prim_g[4], prim[4], pc[4];
    local_frame(bc, cx, cy, prim_w);
    memcpy(prim_g, prim_w, sizeof prim_g);
    int e = get_primary(p, c->W + cell * 4, pc);
    if (e) return e;
    local_frame(pc, cx, cy, prim);
    prim_g[0] = prim[0] / prim[3] * prim_w[3];
    double tau;
    e = get_tau(p, prim_g, &tau);
    if (e) return e;
    double Mt[5];
    time_coeffs(dt, tau, Mt);
    e = face_equilibrium(p, nv, vn, vt, c->w, prim_g, Hg, Bg, rh, rb);
    if (e) return e;
    double qf[2];
    heat_flux(nv, hv, bv, vn, vt, c->w, prim_g, qf);
    shakhov(p, nv, Hg, Bg, vn, vt, qf, prim_g, Hp, Bp);
    double cg[4], cg1[4], sw[4], a_gn[4], a_gt[4], a_T[4];
    get_conserved(p, prim_g, cg);
    local_frame(c->W + cell * 4, cx, cy, cg1);
    for (int m = 0; m < 4; ++m) sw[m] = (cg[m] - cg1[m]) / ((double)side * 0.5 * len);
    micro_slope(p->ck, prim_g, sw, a_gn);
    double swt[4] = {0, 0, 0, 0};
    for (int k = 0; k < nv; ++k) {
        double wk = c->w[k], a = vn[k], t = vt[k], v2 = a * a + t * t;
        swt[0] = swt[0] + wk * sht[k];
        swt[1] = swt[1] + wk * a * sht[k];
        swt[2] = swt[2] + wk * t * sht[k];
        swt[3] = swt[3] + 0.5 * wk * (v2 * sht[k] + sbt[k]);
    }
    micro_slope(p->ck, prim_g, swt, a_gt);
    double Mu[MNUM + 1], MuL[MNUM + 1], MuR[MNUM + 1], Mv[MTUM + 1], Mxi[3], Mau[4], Mbv[4];
    calc_moment(p->ck, prim_g, Mu, Mv, Mxi, MuL, MuR);
    moment_auvxi(a_gn, Mu, Mv, Mxi, 1, 0, Mau);
    moment_auvxi(a_gt, Mu, Mv, Mxi, 0, 1, Mbv);
    for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (Mau[m] + Mbv[m]);
    micro_slope(p->ck, prim_g, sw, a_T);
    double pshape[4] = {1.0, prim_w[1], prim_w[2], prim_w[3]};
    e = face_equilibrium(p, nv, vn, vt, c->w, pshape, Hw, Bw, rh, rb);
    if (e) return e;
    double inc = 0.0, refl = 0.0;
    for (int k = 0; k < nv; ++k) {
        double wk = c->w[k], a = vn[k], t = vt[k];
        double dk = dl[k], ik = 1.0 - dk;
        double slh = a * shn[k] + t * sht[k];
        double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hg[k] + 0.5 * a_gn[3] * ((a * a + t * t) * Hg[k] + Bg[k]);
        double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hg[k] + 0.5 * a_gt[3] * ((a * a + t * t) * Hg[k] + Bg[k]);
        double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hg[k] + 0.5 * a_T[3] * ((a * a + t * t) * Hg[k] + Bg[k]);
        inc = inc + wk * a * ik * (Mt[0] * (Hg[k] + Hp[k]) + Mt[1] * (a * Ha_gn + t * Ha_gt) + Mt[2] * Ha_T +
                                   Mt[3] * hv[k] - Mt[4] * slh);
        refl = refl + wk * a * Hw[k] * dk;
    }
    refl = dt * refl;
    prim_w[0] = -inc / refl;
    for (int k = 0; k < nv; ++k) { Hw[k] = prim_w[0] * Hw[k]; Bw[k] = prim_w[0] * Bw[k]; }
    for (int k = 0; k < nv; ++k) {
        double a = vn[k], t = vt[k], v2 = a * a + t * t;
        double dk = dl[k], ik = 1.0 - dk;
        double Hgk = Hg[k], Bgk = Bg[k];
        double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hgk + 0.5 * a_gn[3] * (v2 * Hgk + Bgk);
        double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hgk + 0.5 * a_gt[3] * (v2 * Hgk + Bgk);
        double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hgk + 0.5 * a_T[3] * (v2 * Hgk + Bgk);
        double Ba_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Bgk + 0.5 * a_gn[3] * (v2 * Bgk + Mxi[2] * Hgk);
        double Ba_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Bgk + 0.5 * a_gt[3] * (v2 * Bgk + Mxi[2] * Hgk);
        double Ba_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Bgk + 0.5 * a_T[3] * (v2 * Bgk + Mxi[2] * Hgk);
        Fh[k] = flen * (dt * a * Hw[k] * dk + Mt[0] * a * (Hgk + Hp[k]) * ik + Mt[1] * a * a * Ha_gn * ik +
                        Mt[1] * a * t * Ha_gt * ik + Mt[2] * a * Ha_T * ik + Mt[3] * a * hv[k] * ik -
                        Mt[4] * a * (a * shn[k] + t * sht[k]) * ik);
        Fb[k] = flen * (dt * a * Bw[k] * dk + Mt[0] * a * (Bgk + Bp[k]) * ik + Mt[1] * a * a * Ba_gn * ik +
                        Mt[1] * a * t * Ba_gt * ik + Mt[2] * a * Ba_T * ik + Mt[3] * a * bv[k] * ik -
                        Mt[4] * a * (a * sbn[k] + t * sbt[k]) * ik);
    }
    double fl[4] = {0, 0, 0, 0};
    for (int k = 0; k < nv; ++k) {
        double hk = Fh[k] / flen, bk = Fb[k] / flen;
        fl[0] = fl[0] + c->w[k] * hk;
        fl[1] = fl[1] + c->w[k] * (vn[k] * hk);
        fl[2] = fl[2] + c->w[k] * (vt[k] * hk);
        fl[3] = fl[3] + c->w[k] * (0.5 * ((vn[k] * vn[k] + vt[k] * vt[k]) * hk + bk));
    }
    aero[0] = fl[1] / dt;
    aero[1] = fl[2] / dt;
    aero[2] = fl[3] / dt - prim_w[2] * fl[2] / dt;
    double g[4];
    global_frame(fl, cx, cy, g);
    for (int m = 0; m < 4; ++m) Fw[m] = flen * g[m];
    return 0;
}

/* EvolutionNative (mod_Evolution.f90:46-177) for x-periodic + two walls. */
typedef struct { uo_ctx* c; double dt; int* err; } evo_arg;

static void evo_body(void* vp, int f, int tid) {
    evo_arg* a = (evo_arg*)vp;
    uo_ctx* c = a->c;
    double dt = a->dt;
    int nx = c->p.nx, ny = c->p.ny, nv = c->p.nvel;
    int nfx = nx * ny, nfy = nx * (ny - 1);
    int e = 0;
    if (f < nfx) {
        int j = f / nx, i = f % nx;
        int cl = j * nx + (i + nx - 1) % nx, cr = j * nx + i;
        size_t o = (size_t)j * nx + i;
        e = interior_face(c, tid, 0, cl, cr, dt, c->fxh + o * nv, c->fxb + o * nv, c->fxw + o * 4);
    } else if (f < nfx + nfy) {
        int g = f - nfx, jf = 1 + g / nx, i = g % nx;
        int cl = (jf - 1) * nx + i, cr = jf * nx + i;
        size_t o = (size_t)jf * nx + i;
        e = interior_face(c, tid, 1, cl, cr, dt, c->fyLh + o * nv, c->fyLb + o * nv, c->fyLw + o * 4);
        memcpy(c->fyRh + o * nv, c->fyLh + o * nv, sizeof(double) * nv);
        memcpy(c->fyRb + o * nv, c->fyLb + o * nv, sizeof(double) * nv);
        memcpy(c->fyRw + o * 4, c->fyLw + o * 4, sizeof(double) * 4);
    } else {
        int g = f - nfx - nfy, i = g % nx;
        if (g < nx) {
            size_t o = (size_t)i;
            e = wall_face(c, tid, -1, i, 0, dt, c->fyLh + o * nv, c->fyLb + o * nv, c->fyLw + o * 4, c->wall_aero + i * 3);
        } else {
            size_t o = (size_t)ny * nx + i;
            e = wall_face(c, tid, +1, (ny - 1) * nx + i, 1, dt, c->fyRh + o * nv, c->fyRb + o * nv, c->fyRw + o * 4,
                          c->wall_aero + (nx + i) * 3);
        }
    }
    a->err[f] = e;
}

/* EvolutionNative (mod_Evolution.f90:46-177) for x-periodic + two walls; faces are independent. */
int uo_evolution(uo_ctx* c, double dt) {
    int nx = c->p.nx, ny = c->p.ny;
    int ntot = nx * ny + nx * (ny - 1) + 2 * nx;
    int* err = (int*)calloc((size_t)ntot, sizeof(int));
    evo_arg a = {c, dt, err};
    par_for(ntot, evo_body, &a, g_threads < c->nthr ? g_threads : c->nthr);
    int e = 0;
    for (int f = 0; f < ntot && !e; ++f) e = err[f];
    free(err);
    return e;
}

/* ------------------------------------------------------------------ residual + update */

/* ComputeResidual (mod_Residual.f90:17-132) for the unified low-order path:
 * AssembleMacroResidual, AssembleMicroFluxResidual, AssembleSteadyRateResiduals with the
 * EnforceStreamingMomentCompatibility projection (mod_ImplicitMicro.f90:293-306) and, when
 * with_collision, the physical equilibrium/collision used by the implicit paths. */
typedef struct { uo_ctx* c; double dt; int with_collision; } res_arg;

static void residual_body(void* vp, int cc, int tid) {
    res_arg* a = (res_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    double dt = a->dt;
    int with_collision = a->with_collision;
    int nx = p->nx, nv = p->nvel;
    double area_inv = 1.0 / c->area;
    double dti = 1.0 / dt;
    {
        double** T = scratch_t(c, tid);
        int j = cc / nx, i = cc % nx;
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
        for (int m = 0; m < 4; ++m) c->rate_w[cc * 4 + m] = c->res_w[cc * 4 + m] * dti;
        for (int k = 0; k < nv; ++k) {
            c->stream_h[(size_t)cc * nv + k] = c->res_h[(size_t)cc * nv + k] * dti;
            c->stream_b[(size_t)cc * nv + k] = c->res_b[(size_t)cc * nv + k] * dti;
        }
        int e = 0;
        if (!uo_project_moments(nv, c->stream_h + (size_t)cc * nv, c->stream_b + (size_t)cc * nv, c->rate_w + cc * 4,
                                c->u, c->v, c->w, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv))
            e = 444;
        for (int k = 0; k < nv; ++k) {
            c->res_h[(size_t)cc * nv + k] = c->stream_h[(size_t)cc * nv + k] * dt;
            c->res_b[(size_t)cc * nv + k] = c->stream_b[(size_t)cc * nv + k] * dt;
        }
        if (with_collision && !e) {
            double prim[4], tau, q[2];
            e = get_primary(p, c->W + cc * 4, prim);
            if (!e) e = get_tau(p, prim, &tau);
            if (!e) {
                const double *h = c->h + (size_t)cc * nv, *b = c->b + (size_t)cc * nv;
                double *eh = c->peq_h + (size_t)cc * nv, *eb = c->peq_b + (size_t)cc * nv;
                heat_flux(nv, h, b, c->u, c->v, c->w, prim, q);
                maxwell(p, nv, c->u, c->v, prim, eh, eb);
                shakhov(p, nv, eh, eb, c->u, c->v, q, prim, T[0], T[1]);
                for (int k = 0; k < nv; ++k) { eh[k] = eh[k] + T[0][k]; eb[k] = eb[k] + T[1][k]; }
                memcpy(T[2], eh, sizeof(double) * nv);
                memcpy(T[3], eb, sizeof(double) * nv);
                if (!uo_project_moments(nv, eh, eb, c->W + cc * 4, c->u, c->v, c->w, T[2], T[3])) e = 444;
                for (int k = 0; k < nv; ++k) {
                    c->pcol_h[(size_t)cc * nv + k] = (eh[k] - h[k]) / tau;
                    c->pcol_b[(size_t)cc * nv + k] = (eb[k] - b[k]) / tau;
                }
            }
        }
        c->cell_err[cc] = e;
    }
}

int uo_compute_residual(uo_ctx* c, double dt, int with_collision) {
    res_arg a = {c, dt, with_collision};
    par_for(c->nc, residual_body, &a, g_threads < c->nthr ? g_threads : c->nthr);
    /* first failing cell in cell order, like the reference's per-rank loop order */
    for (int cc = 0; cc < c->nc; ++cc) if (c->cell_err[cc]) return c->cell_err[cc];
    return 0;
}

/* ApplyExplicitUpdate + ApplyMicroExplicitUpdate + residual norms
 * (mod_TimeIntegrator.f90:16-134,163-191,235-293).  Cells update in parallel; the residual-norm
 * terms are stored per cell and summed afterwards in cell order, as the single-rank loop does. */
typedef struct { uo_ctx* c; double dt; } upd_arg;

static void update_body(void* vp, int cc, int tid) {
    upd_arg* a = (upd_arg*)vp;
    uo_ctx* c = a->c;
    const uo_params* p = &c->p;
    double dt = a->dt;
    int nv = p->nvel;
    {
        double** T = scratch_t(c, tid);
        double *Ho = T[17], *Bo = T[18], *Hn = T[19], *Bn = T[20], *Hp = T[21], *Bp = T[22];
        double *rh = T[13], *rb = T[14];
        double Wold[4], po[4], pn[4], to, tn;
        double* dg = c->cell_diag + (size_t)cc * 13;
        int e = 0;
        memcpy(Wold, c->W + cc * 4, sizeof Wold);
        e = get_primary(p, Wold, po);
        if (!e) { maxwell(p, nv, c->u, c->v, po, Ho, Bo); e = get_tau(p, po, &to); }
        if (!e) {
            for (int m = 0; m < 4; ++m) c->W[cc * 4 + m] = c->W[cc * 4 + m] + c->res_w[cc * 4 + m];
            for (int m = 0; m < 4; ++m) if (!isfinite(c->W[cc * 4 + m])) e = 4;
        }
        if (!e) e = get_primary(p, c->W + cc * 4, pn);
        if (!e) { maxwell(p, nv, c->u, c->v, pn, Hn, Bn); e = get_tau(p, pn, &tn); }
        if (!e) {
            for (int m = 0; m < 4; ++m) {
                double d = (Wold[m] - c->W[cc * 4 + m]) * c->area / dt;
                dg[m] = d * d;
                dg[9 + m] = fabs(d);
                dg[4 + m] = fabs(c->W[cc * 4 + m]) * c->area;
            }
            dg[8] = c->area * c->area;
            double* h = c->h + (size_t)cc * nv;
            double* b = c->b + (size_t)cc * nv;
            double qf[2];
            heat_flux(nv, h, b, c->u, c->v, c->w, po, qf);
            shakhov(p, nv, Ho, Bo, c->u, c->v, qf, po, Hp, Bp);
            for (int k = 0; k < nv; ++k) { Ho[k] = Ho[k] + Hp[k]; Bo[k] = Bo[k] + Bp[k]; }
            shakhov(p, nv, Hn, Bn, c->u, c->v, qf, pn, Hp, Bp);
            for (int k = 0; k < nv; ++k) { Hn[k] = Hn[k] + Hp[k]; Bn[k] = Bn[k] + Bp[k]; }
            double tg[4];
            get_conserved(p, po, tg);
            memcpy(rh, Ho, sizeof(double) * nv); memcpy(rb, Bo, sizeof(double) * nv);
            if (!uo_project_moments(nv, Ho, Bo, tg, c->u, c->v, c->w, rh, rb)) e = 444;
            memcpy(rh, Hn, sizeof(double) * nv); memcpy(rb, Bn, sizeof(double) * nv);
            if (!e && !uo_project_moments(nv, Hn, Bn, c->W + cc * 4, c->u, c->v, c->w, rh, rb)) e = 444;
            if (!e) {
                double inv = 1.0 / (1.0 + 0.5 * dt / tn);
                const double *fh = c->res_h + (size_t)cc * nv, *fb = c->res_b + (size_t)cc * nv;
                for (int k = 0; k < nv; ++k) {
                    double ho = h[k], bo = b[k];
                    h[k] = (ho + fh[k] + 0.5 * dt * (Hn[k] / tn + (Ho[k] - ho) / to)) * inv;
                    b[k] = (bo + fb[k] + 0.5 * dt * (Bn[k] / tn + (Bo[k] - bo) / to)) * inv;
                }
            }
        }
        c->cell_err[cc] = e;
    }
}

int uo_apply_explicit_update(uo_ctx* c, double dt, double* res_out) {
    const uo_params* p = &c->p;
    upd_arg a = {c, dt};
    par_for(c->nc, update_body, &a, g_threads < c->nthr ? g_threads : c->nthr);
    for (int cc = 0; cc < c->nc; ++cc) if (c->cell_err[cc]) return c->cell_err[cc];
    double sumRes[4] = {0, 0, 0, 0}, sumAvg[4] = {0, 0, 0, 0}, areaSq = 0.0, maxCell[4] = {0, 0, 0, 0};
    for (int cc = 0; cc < c->nc; ++cc) {
        const double* dg = c->cell_diag + (size_t)cc * 13;
        for (int m = 0; m < 4; ++m) {
            if (dg[9 + m] > maxCell[m]) maxCell[m] = dg[9 + m];
            sumRes[m] = sumRes[m] + dg[m];
        }
        for (int m = 0; m < 4; ++m) sumAvg[m] = sumAvg[m] + dg[4 + m];
        areaSq = areaSq + dg[8];
    }
    /* residual norms (mod_TimeIntegrator.f90:102-127) */
    double ncell = (double)(p->nx * p->ny);
    double num[4], den[4], rel[4], absr[4], res[4];
    for (int m = 0; m < 4; ++m) {
        num[m] = sqrt(ncell * sumRes[m]);
        den[m] = sumAvg[m] + SMV;
        rel[m] = num[m] / den[m];
        absr[m] = sqrt(sumRes[m] / fmax(areaSq, SMV));
    }
    double ords = fmax(fmax(sumAvg[0], sumAvg[3]), SMV);
    for (int m = 0; m < 4; ++m) {
        int near0 = sumAvg[m] <= sqrt(DBL_EPSILON) * fmax(ords, DBL_MIN);
        res[m] = near0 ? absr[m] : rel[m];
        if (!isfinite(res[m])) return 8;
    }
    if (res_out) memcpy(res_out, res, sizeof res);
    return 0;
}

int uo_explicit_step(uo_ctx* c, double* dt_out, double* res_out) {
    double dt = uo_timestep(c);
    if (!isfinite(dt)) return 101;
    if (dt_out) *dt_out = dt;
    uo_interpolation(c);
    int e = uo_evolution(c, dt);
    if (e) return e;
    e = uo_compute_residual(c, dt, 0);
    if (e) return e;
    return uo_apply_explicit_update(c, dt, res_out);
}

/* ================================================================== ImplicitSteady
 * mod_SteadyImplicit.f90:379-462 with the closed-Couette mass rescale (mod_ClosedCouetteMass.f90)
 * and the accepted-state re-evaluation (mod_R5Observe.f90:287-358).  The reference runs on NP_Y
 * ranks stacked in y (nslab here); PR(2) and LU-SGS are Gauss-Seidel inside a rank and read the
 * other ranks' corrections (and the x-periodic self-exchange) from halos refreshed only at the
 * exchange points, so the emulation keeps a halo snapshot (dw_ghost, dh_ghost) refreshed at
 * exactly those points. */

static int uo_is_physical(const double w[4]) {            /* IsPhysicalState (mod_ImplicitCommon.f90:10-20) */
    for (int m = 0; m < 4; ++m) if (!isfinite(w[m])) return 0;
    if (w[0] <= 0.0) return 0;
    double e = w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0];
    return isfinite(e) && e > 0.0;
}

static void euler_flux(double gamma, const double w[4], double nx, double ny, double f[4]) {   /* EulerFluxNormal */
    double u = w[1] / w[0], v = w[2] / w[0], un = u * nx + v * ny;
    double p = (gamma - 1.0) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    f[0] = w[0] * un;
    f[1] = w[1] * un + p * nx;
    f[2] = w[2] * un + p * ny;
    f[3] = (w[3] + p) * un;
}

static void zhu_map(const double w[4], double uw, double vw, double g[4]) {  /* ZhuMovingWallMap (mod_ImplicitBoundary.f90:187-194) */
    g[0] = w[0];
    g[1] = 2.0 * uw * w[0] - w[1];
    g[2] = 2.0 * vw * w[0] - w[2];
    g[3] = w[3] + 2.0 * (uw * uw + vw * vw) * w[0] - 2.0 * uw * w[1] - 2.0 * vw * w[2];
}

static int slab_rows(const uo_ctx* c) { return c->p.ny / (c->p.nslab > 0 ? c->p.nslab : 1); }
static int same_slab(const uo_ctx* c, int j0, int j1) { return j0 / slab_rows(c) == j1 / slab_rows(c); }

/* Face geometry of GetFaceGeometry (mod_ImplicitMacro.f90:236-263): face 0..3 = left, right,
 * bottom, top; outward normal, face length, neighbour cell, and whether the neighbour is read from
 * the halo (other rank or the x-periodic self-exchange) or is a physical wall. */
typedef struct { double nx, ny, len; int nb; int ghost; int wall; double dist; } face_geo;

static face_geo uo_face(const uo_ctx* c, int i, int j, int f) {
    const uo_params* p = &c->p;
    face_geo g;
    int nx = p->nx, ny = p->ny;
    double xi = (i + 0.5) * p->dx, yj = (j + 0.5) * p->dy;
    g.wall = 0; g.ghost = 0;
    if (f == 0) {
        g.nx = -1.0; g.ny = 0.0; g.len = p->dy;
        int ni = i - 1; g.ghost = ni < 0; if (ni < 0) ni += nx;
        g.nb = j * nx + ni;
        /* ghost centres on the outer ranks are re-extrapolated after the periodic copy
         * (mod_InitializeFlow.f90:418-446), so the seam distance is one cell as well */
        g.dist = fabs(((i - 1 + 0.5) * p->dx - xi) * g.nx + 0.0);
    } else if (f == 1) {
        g.nx = 1.0; g.ny = -0.0; g.len = p->dy;
        int ni = i + 1; g.ghost = ni >= nx; if (ni >= nx) ni -= nx;
        g.nb = j * nx + ni;
        g.dist = fabs(((i + 1 + 0.5) * p->dx - xi) * g.nx + 0.0);
    } else if (f == 2) {
        g.nx = 0.0; g.ny = -1.0; g.len = p->dx;
        if (j == 0) { g.wall = 1; g.nb = -1; g.dist = p->dy; }
        else { g.nb = (j - 1) * nx + i; g.ghost = !same_slab(c, j, j - 1); g.dist = fabs(0.0 + (((j - 1) + 0.5) * p->dy - yj) * g.ny); }
    } else {
        g.nx = -0.0; g.ny = 1.0; g.len = p->dx;
        if (j == ny - 1) { g.wall = 1; g.nb = -1; g.dist = p->dy; }
        else { g.nb = (j + 1) * nx + i; g.ghost = !same_slab(c, j, j + 1); g.dist = fabs(0.0 + (((j + 1) + 0.5) * p->dy - yj) * g.ny); }
    }
    return g;
}

/* ImplicitSpectralRadius (mod_ImplicitMacro.f90:15-55) */
static double spectral_radius(const uo_ctx* c, const double wi[4], const double wj[4], const face_geo* g) {
    const uo_params* p = &c->p;
    double pi_[4], pj[4], ti, tj;
    if (get_primary(p, wi, pi_) || get_primary(p, wj, pj)) return NAN;
    double rho_avg = 0.5 * (pi_[0] + pj[0]);
    double u_avg = 0.5 * (pi_[1] + pj[1]);
    double v_avg = 0.5 * (pi_[2] + pj[2]);
    double p_i = 0.5 * pi_[0] / pi_[3], p_j = 0.5 * pj[0] / pj[3];
    double p_avg = 0.5 * (p_i + p_j);
    if (get_tau(p, pi_, &ti) || get_tau(p, pj, &tj)) return NAN;
    double mu_avg = 0.5 * (ti * p_i + tj * p_j);
    double sos = sqrt(p->gamma * p_avg / rho_avg);
    return fabs(u_avg * g->nx + v_avg * g->ny) + sos + 2.0 * mu_avg / (rho_avg * fmax(g->dist, 1000.0 * DBL_EPSILON));
}

/* RelaxMacroPoint (mod_ImplicitMacro.f90:90-123) */
static int relax_macro(uo_ctx* c, int i, int j, double dt_pseudo) {
    const uo_params* p = &c->p;
    int cc = j * p->nx + i;
    double sdt[4] = {0, 0, 0, 0}, sgn[4] = {0, 0, 0, 0}, sg = 0.0;
    for (int f = 0; f < 4; ++f) {
        face_geo g = uo_face(c, i, j, f);
        const double* wi = c->W + cc * 4;
        double wj[4], dnb[4], fn[4], fo[4], dti[4], dtj[4], t[4];
        if (g.wall) {
            double uw = p->wall_ux[f == 2 ? 0 : 1], vw = 0.0;
            zhu_map(wi, uw, vw, wj);
            zhu_map(c->dw + cc * 4, uw, vw, dnb);
        } else {
            memcpy(wj, c->W + g.nb * 4, sizeof wj);
            memcpy(dnb, (g.ghost ? c->dw_ghost : c->dw) + g.nb * 4, sizeof dnb);
        }
        for (int m = 0; m < 4; ++m) t[m] = wi[m] + c->dw[cc * 4 + m];
        euler_flux(p->gamma, t, g.nx, g.ny, fn);
        euler_flux(p->gamma, wi, g.nx, g.ny, fo);
        for (int m = 0; m < 4; ++m) dti[m] = fn[m] - fo[m];
        for (int m = 0; m < 4; ++m) t[m] = wj[m] + dnb[m];
        euler_flux(p->gamma, t, g.nx, g.ny, fn);
        euler_flux(p->gamma, wj, g.nx, g.ny, fo);
        for (int m = 0; m < 4; ++m) dtj[m] = fn[m] - fo[m];
        double gam = spectral_radius(c, wi, wj, &g);
        if (!isfinite(gam) || !(gam > 0.0)) return 0;
        for (int m = 0; m < 4; ++m) {
            double s = dti[m] + dtj[m];
            if (!isfinite(s)) return 0;
            sdt[m] = sdt[m] + g.len * s;
            sgn[m] = sgn[m] + g.len * gam * dnb[m];
        }
        sg = sg + g.len * gam;
    }
    double diag = 1.0 / dt_pseudo + 0.5 * sg / c->area;
    double rhs[4];
    for (int m = 0; m < 4; ++m)
        rhs[m] = c->rate_w[cc * 4 + m] - 0.5 * 1.0 * sdt[m] / c->area + 0.5 * 1.0 * sgn[m] / c->area;
    if (!(isfinite(diag) && diag > 0.0)) return 0;
    for (int m = 0; m < 4; ++m) if (!isfinite(rhs[m])) return 0;
    for (int m = 0; m < 4; ++m) c->dw[cc * 4 + m] = rhs[m] / diag;
    return 1;
}

/* SolveMacroPR2 (mod_ImplicitMacro.f90:57-88) over nslab ranks */
static int solve_macro_pr2(uo_ctx* c, double dt_pseudo) {
    const uo_params* p = &c->p;
    int rows = slab_rows(c), nx = p->nx;
    memcpy(c->dw_ghost, c->dw, sizeof(double) * c->nc * 4);    /* MPIExchangeDeltaMacro */
    for (int sweep = 0; sweep < p->macro_sweeps; ++sweep) {
        for (int s = 0; s < p->nslab; ++s) {
            for (int j = s * rows; j < (s + 1) * rows; ++j)
                for (int i = 0; i < nx; ++i) if (!relax_macro(c, i, j, dt_pseudo)) return 0;
            for (int j = (s + 1) * rows - 1; j >= s * rows; --j)
                for (int i = nx - 1; i >= 0; --i) if (!relax_macro(c, i, j, dt_pseudo)) return 0;
        }
        memcpy(c->dw_ghost, c->dw, sizeof(double) * c->nc * 4);
    }
    for (int m = 0; m < c->nc * 4; ++m) if (!isfinite(c->dw[m])) return 0;
    return 1;
}

/* ComputeDiffuseWallFaceDelta (mod_ImplicitBoundary.f90:282-326) for the wall face of cell cc:
 * returns delta_rho (the reflected face correction is delta_rho * h_unit for vn < 0). */
static int wall_delta_rho(uo_ctx* c, int cc, int top, double* drho) {
    const uo_params* p = &c->p;
    int nv = p->nvel;
    double nxo = top ? -0.0 : 0.0, nyo = top ? 1.0 : -1.0;
    double bc[4] = {1.0, p->wall_ux[top], 0.0, 1.0 / p->wall_tnative[top]}, pl[4];
    local_frame(bc, nxo, nyo, pl);
    pl[0] = 1.0;
    double inc = 0.0, refl = 0.0, outs = 0.0;
    for (int k = 0; k < nv; ++k) {
        double vn = c->u[k] * nxo + c->v[k] * nyo, vt = -c->u[k] * nyo + c->v[k] * nxo;
        double sel = vn < 0.0 ? 1.0 : 0.0;
        double dvn = vn - pl[1], dvt = vt - pl[2];
        double hu = pl[0] * (pl[3] / PI_D) * exp(-pl[3] * (dvn * dvn + dvt * dvt));
        inc += c->w[k] * vn * c->dh[(size_t)cc * nv + k] * (1.0 - sel);
        refl += c->w[k] * vn * hu * sel;
        outs += fabs(c->w[k] * vn * hu * sel);
    }
    if (fabs(refl) <= 1000.0 * DBL_EPSILON * fmax(outs, DBL_MIN)) return 0;
    *drho = -inc / refl;
    return 1;
}

/* One LU-SGS stage over one slab (SolveMicroLUSGS / RelaxMicroPoint, mod_ImplicitMicro.f90:366-487) */
static int lusgs_stage(uo_ctx* c, int s, int backward, double dt_pseudo) {
    const uo_params* p = &c->p;
    int nv = p->nvel, nx = p->nx, ny = p->ny, rows = slab_rows(c);
    for (int jj = 0; jj < rows; ++jj) {
        int j = backward ? (s + 1) * rows - 1 - jj : s * rows + jj;
        for (int ii = 0; ii < nx; ++ii) {
            int i = backward ? nx - 1 - ii : ii;
            int cc = j * nx + i;
            /* frozen wall closure from this cell's correction at the start of its velocity loop */
            double drho[2] = {0.0, 0.0};
            int haswall[2] = {j == 0, j == ny - 1};
            for (int t = 0; t < 2; ++t)
                if (haswall[t] && !wall_delta_rho(c, cc, t, &drho[t])) return 0;
            face_geo g[4];
            for (int f = 0; f < 4; ++f) g[f] = uo_face(c, i, j, f);
            for (int kk = 0; kk < nv; ++kk) {
                int k = backward ? nv - 1 - kk : kk;
                size_t q = (size_t)cc * nv + k;
                double rhs_h = c->stream_h[q] + (c->eq_h[q] - c->h[q]) / c->tau_t[cc];
                double rhs_b = c->stream_b[q] + (c->eq_b[q] - c->b[q]) / c->tau_t[cc];
                if (p->high_order) {   /* mod_ImplicitMicro.f90:467-470 */
                    rhs_h = rhs_h + c->pcol_h[q] - c->lco_h[q];
                    rhs_b = rhs_b + c->pcol_b[q] - c->lco_b[q];
                }
                double diag = 1.0 / dt_pseudo + 1.0 / c->tau_t[cc];
                for (int f = 0; f < 4; ++f) {
                    double un = c->u[k] * g[f].nx + c->v[k] * g[f].ny;
                    double nh, nb;
                    if (g[f].wall) {
                        int top = f == 3;
                        double nxo = top ? -0.0 : 0.0, nyo = top ? 1.0 : -1.0;
                        double vn = c->u[k] * nxo + c->v[k] * nyo, vt = -c->u[k] * nyo + c->v[k] * nxo;
                        double bc[4] = {1.0, p->wall_ux[top], 0.0, 1.0 / p->wall_tnative[top]}, pl[4];
                        local_frame(bc, nxo, nyo, pl);
                        double dvn = vn - pl[1], dvt = vt - pl[2];
                        double hu = 1.0 * (pl[3] / PI_D) * exp(-pl[3] * (dvn * dvn + dvt * dvt));
                        double bu = hu * ((double)p->ck / (2.0 * pl[3]));
                        double sel = vn < 0.0 ? 1.0 : 0.0;
                        nh = drho[top] * hu * sel + c->dh[q] * (1.0 - sel);
                        nb = drho[top] * bu * sel + c->db[q] * (1.0 - sel);
                    } else {
                        size_t qn = (size_t)g[f].nb * nv + k;
                        nh = g[f].ghost ? c->dh_ghost[qn] : c->dh[qn];
                        nb = g[f].ghost ? c->db_ghost[qn] : c->db[qn];
                    }
                    diag = diag + 1.0 * fmax(un, 0.0) * g[f].len / c->area;
                    rhs_h = rhs_h - 1.0 * fmin(un, 0.0) * g[f].len * nh / c->area;
                    rhs_b = rhs_b - 1.0 * fmin(un, 0.0) * g[f].len * nb / c->area;
                }
                if (!(diag > 0.0 && isfinite(diag) && isfinite(rhs_h) && isfinite(rhs_b))) return 0;
                c->dh[q] = rhs_h / diag;
                c->db[q] = rhs_b / diag;
            }
        }
    }
    return 1;
}

/* UpdateImplicitResidualDiagnostics (mod_ImplicitDiagnostics.f90:223-322); sci[22] = SciencePack
 * (mod_R5Observe.f90:27-32) plus r5 raw values; sums taken per slab then over slabs. */
static void implicit_diagnostics(uo_ctx* c, double dt, double sci[22]) {
    const uo_params* p = &c->p;
    int nv = p->nvel, nx = p->nx, rows = slab_rows(c);
    double num[4] = {0}, den[4] = {0}, wgt = 0, mic[4] = {0}, mass = 0;
    for (int s = 0; s < p->nslab; ++s) {
        double ln[4] = {0}, ld[4] = {0}, lw = 0, lm[4] = {0}, lmass = 0;
        for (int j = s * rows; j < (s + 1) * rows; ++j)
            for (int i = 0; i < nx; ++i) {
                int cc = j * nx + i;
                for (int m = 0; m < 4; ++m) {
                    double a = c->area * c->rate_w[cc * 4 + m];
                    ln[m] = ln[m] + a * a;
                    ld[m] = ld[m] + c->area * fabs(c->W[cc * 4 + m] + dt * c->rate_w[cc * 4 + m]);
                }
                lw = lw + c->area * c->area;
                double s3 = 0.0, s4 = 0.0;
                for (int k = 0; k < nv; ++k) {
                    size_t q = (size_t)cc * nv + k;
                    double dh = c->stream_h[q] + c->pcol_h[q], db = c->stream_b[q] + c->pcol_b[q];
                    lm[0] = lm[0] + c->area * c->w[k] * dh * dh;
                    lm[1] = lm[1] + c->area * c->w[k] * db * db;
                    s3 += c->w[k] * fmax(c->h[q] * c->h[q], c->peq_h[q] * c->peq_h[q]);
                    s4 += c->w[k] * fmax(c->b[q] * c->b[q], c->peq_b[q] * c->peq_b[q]);
                }
                lm[2] = lm[2] + c->area * s3;
                lm[3] = lm[3] + c->area * s4;
                lmass = lmass + c->rate_w[cc * 4] * c->area;
            }
        for (int m = 0; m < 4; ++m) { num[m] += ln[m]; den[m] += ld[m]; mic[m] += lm[m]; }
        wgt += lw; mass += lmass;
    }
    double rel[4], absr[4], res[4];
    double ncell = (double)(p->nx * p->ny);
    for (int m = 0; m < 4; ++m) {
        rel[m] = sqrt(ncell * num[m]) / (den[m] + SMV);
        absr[m] = sqrt(num[m] / fmax(wgt, SMV));
    }
    double raw_h = sqrt(mic[0]), raw_b = sqrt(mic[1]);
    double ords = fmax(fmax(den[0], den[3]), SMV);
    for (int m = 0; m < 4; ++m) res[m] = (den[m] <= sqrt(DBL_EPSILON) * fmax(ords, DBL_MIN)) ? absr[m] : rel[m];
    double h_raw = sqrt(mic[0] / fmax(mic[2], SMV)), b_raw = sqrt(mic[1] / fmax(mic[3], SMV));
    if (!c->ref_init) { c->ref_h = h_raw; c->ref_b = b_raw; c->ref_init = 1; }
    double h_rel = c->ref_h > DBL_MIN ? h_raw / c->ref_h : h_raw;
    double b_rel = c->ref_b > DBL_MIN ? b_raw / c->ref_b : b_raw;
    double nzr = fmax(100.0 * p->residual_tol, 1000.0 * DBL_EPSILON);
    double h_norm = c->ref_h <= nzr ? h_raw : h_raw / c->ref_h;
    double b_norm = c->ref_b <= nzr ? b_raw : b_raw / c->ref_b;
    for (int m = 0; m < 4; ++m) { sci[m] = res[m]; sci[4 + m] = rel[m]; sci[8 + m] = absr[m]; }
    sci[12] = h_norm; sci[13] = b_norm; sci[14] = h_rel; sci[15] = b_rel; sci[16] = h_raw; sci[17] = b_raw;
    sci[18] = 0.0;   /* implicit_moment_error: filled by the caller */
    sci[19] = fabs(mass); sci[20] = raw_h; sci[21] = raw_b;
}

/* MassStatistics (mod_ClosedCouetteMass.f90:173-204): totals[5], metrics[5] */
static int mass_statistics(uo_ctx* c, double totals[5], double metrics[5]) {
    const uo_params* p = &c->p;
    int nv = p->nvel, nx = p->nx, rows = slab_rows(c);
    int ok = 1;
    double t[5] = {0}, mx[3] = {0}, mn[2] = {INFINITY, INFINITY};
    for (int s = 0; s < p->nslab; ++s) {
        double lt[5] = {0};
        for (int j = s * rows; j < (s + 1) * rows; ++j)
            for (int i = 0; i < nx; ++i) {
                int cc = j * nx + i;
                double mm[4];
                const double *h = c->h + (size_t)cc * nv, *b = c->b + (size_t)cc * nv, *W = c->W + cc * 4;
                moment_conserved(nv, h, b, c->u, c->v, c->w, mm);
                for (int k = 0; k < nv; ++k) ok &= isfinite(h[k]) && isfinite(b[k]);
                ok &= uo_is_physical(W) && uo_is_physical(mm);
                for (int m = 0; m < 4; ++m) lt[m] = lt[m] + c->area * W[m];
                lt[4] = lt[4] + c->area * mm[0];
                double e1 = 0.0;
                for (int m = 0; m < 4; ++m) e1 = fmax(e1, fabs(W[m] - mm[m]) / fmax(fabs(W[m]), 1.0));
                mx[0] = fmax(mx[0], e1);
                double nh1 = 0, nh2 = 0, nb1 = 0, nb2 = 0;
                for (int k = 0; k < nv; ++k) {
                    nh1 += c->w[k] * fmax(-h[k], 0.0); nh2 += c->w[k] * fabs(h[k]);
                    nb1 += c->w[k] * fmax(-b[k], 0.0); nb2 += c->w[k] * fabs(b[k]);
                }
                mx[1] = fmax(mx[1], nh1 / fmax(nh2, DBL_MIN));
                mx[2] = fmax(mx[2], nb1 / fmax(nb2, DBL_MIN));
                if (isfinite(W[0]) && W[0] > 0.0) {
                    double e = W[3] - 0.5 * (W[1] * W[1] + W[2] * W[2]) / W[0];
                    mn[0] = fmin(mn[0], W[0]); mn[1] = fmin(mn[1], e);
                }
            }
        for (int m = 0; m < 5; ++m) t[m] += lt[m];
    }
    memcpy(totals, t, sizeof t);
    metrics[0] = mx[0]; metrics[1] = mx[1]; metrics[2] = mx[2]; metrics[3] = mn[0]; metrics[4] = mn[1];
    return ok && metrics[0] <= p->moment_tol;
}

/* AssembleSteadyRateResiduals' rate/stream part run again on the cached residuals (the second call
 * inside ApplyOriginalSteadyImplicitUpdate, mod_SteadyImplicit.f90:406, and after ComputeResidual
 * in PhysicalDiagnostic): rate_w, stream_* from res_*, streaming projection, res_* = stream*dt. */
static int reassemble_rates(uo_ctx* c, double dt) {
    int nv = c->p.nvel;
    double dti = 1.0 / dt;
    int ok = 1;
    for (int cc = 0; cc < c->nc; ++cc) {
        for (int m = 0; m < 4; ++m) c->rate_w[cc * 4 + m] = c->res_w[cc * 4 + m] * dti;
        for (int k = 0; k < nv; ++k) {
            c->stream_h[(size_t)cc * nv + k] = c->res_h[(size_t)cc * nv + k] * dti;
            c->stream_b[(size_t)cc * nv + k] = c->res_b[(size_t)cc * nv + k] * dti;
        }
        ok &= uo_project_moments(nv, c->stream_h + (size_t)cc * nv, c->stream_b + (size_t)cc * nv, c->rate_w + cc * 4,
                                 c->u, c->v, c->w, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv);
        for (int k = 0; k < nv; ++k) {
            c->res_h[(size_t)cc * nv + k] = c->stream_h[(size_t)cc * nv + k] * dt;
            c->res_b[(size_t)cc * nv + k] = c->stream_b[(size_t)cc * nv + k] * dt;
        }
    }
    return ok;
}

/* InitializeClosedMass (mod_ClosedCouetteMass.f90:212-241): persistent M0 of the cold start. */
int uo_implicit_init(uo_ctx* c) {
    double t[5], m[5];
    if (!mass_statistics(c, t, m)) return 941;
    c->m0 = t[0];
    c->ref_init = 0;
    c->streak = 0;
    c->mass_scale = 1.0;
    return 0;
}

/* One accepted ImplicitSteady pseudo-step of Solve_UGKS (mod_Solve.f90:84-293) with
 * ClosedCouetteMassRescale: out[] = the sparse_residual.csv row of the accepted state
 * [0] original_gate, [1] moment, [2] M_W, [3] M_h, [4..11] R1..R8, [12..33] science_1..22,
 * [34..49] flux_1..16, [50] reference_h, [51] reference_b, [52] c_minus_1, then extras:
 * [53] alpha, [54] macro_alpha, [55] dt, [56] verified streak, [57..78] science of the
 * pre-update evaluation (the "Implicit iter=" line of the next step prints these). */
int uo_implicit_step(uo_ctx* c, double* out, int nout) {
    const uo_params* p = &c->p;
    int nv = p->nvel, e;
    double row[80];
    memset(row, 0, sizeof row);
    /* TimeStep, Interpolation, Evolution, ComputeResidual (mod_Solve.f90:95-117) */
    double dt = uo_timestep(c);
    if (!isfinite(dt)) return 101;
    c->dt = dt;
    if (p->high_order) {   /* S2NativeEvolution; Interpolation is skipped (mod_Solve.f90:108) */
        if ((e = uo_s2_evolution(c, dt))) return e;
        if ((e = uo_s2_compute_residual(c, dt, 0))) return e;
    } else {
        uo_interpolation(c);
        if ((e = uo_evolution(c, dt))) return e;
        if ((e = uo_compute_residual(c, dt, 1))) return e;
    }
    /* ApplySteadyImplicitUpdate -> ApplyOriginalSteadyImplicitUpdate (mod_SteadyImplicit.f90:379-462) */
    size_t S = (size_t)c->nc * nv;
    memcpy(c->save_h, c->h, S * sizeof(double));
    memcpy(c->save_b, c->b, S * sizeof(double));
    memcpy(c->save_W, c->W, (size_t)c->nc * 4 * sizeof(double));
    if (p->high_order) { if ((e = uo_s2_compute_residual(c, dt, 1))) return e; }
    else if (!reassemble_rates(c, dt)) return 444;
    double sci0[22];
    implicit_diagnostics(c, dt, sci0);
    memcpy(row + 57, sci0, sizeof sci0);
    double dtp = dt * p->ncfl / p->cfl;                     /* PseudoTimeStep */
    memset(c->dw, 0, sizeof(double) * c->nc * 4);             /* ResetImplicitCorrections */
    memset(c->dh, 0, S * sizeof(double));
    memset(c->db, 0, S * sizeof(double));
    if (!solve_macro_pr2(c, dtp)) return 420;
    /* BuildPredictedMacroState (mod_ImplicitMacro.f90:159-185) */
    double malpha = 1.0;
    for (;;) {
        int ok = 1;
        for (int cc = 0; cc < c->nc && ok; ++cc) {
            double t[4];
            for (int m = 0; m < 4; ++m) t[m] = c->W[cc * 4 + m] + malpha * c->dw[cc * 4 + m];
            ok = uo_is_physical(t);
        }
        if (ok) break;
        malpha = 0.5 * malpha;
        if (malpha < p->min_alpha) return 421;
    }
    for (int m = 0; m < c->nc * 4; ++m) c->dw[m] = malpha * c->dw[m];
    for (int m = 0; m < c->nc * 4; ++m) c->wt[m] = c->W[m] + c->dw[m];
    /* BuildPredictedEquilibrium (mod_ImplicitMicro.f90:43-88), low-order branch */
    for (int cc = 0; cc < c->nc; ++cc) {
        double po[4], pt[4], q[2];
        if ((e = get_primary(p, c->W + cc * 4, po))) return e;
        heat_flux(nv, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv, c->u, c->v, c->w, po, q);
        if ((e = get_primary(p, c->wt + cc * 4, pt))) return e;
        if ((e = get_tau(p, pt, &c->tau_t[cc]))) return e;
        double *eh = c->eq_h + (size_t)cc * nv, *eb = c->eq_b + (size_t)cc * nv;
        double** T = scratch_t(c, 0);
        maxwell(p, nv, c->u, c->v, pt, eh, eb);
        shakhov(p, nv, eh, eb, c->u, c->v, q, pt, T[0], T[1]);
        for (int k = 0; k < nv; ++k) { eh[k] = eh[k] + T[0][k]; eb[k] = eb[k] + T[1][k]; }
        memcpy(T[2], eh, sizeof(double) * nv);
        memcpy(T[3], eb, sizeof(double) * nv);
        if (!uo_project_moments(nv, eh, eb, c->wt + cc * 4, c->u, c->v, c->w, T[2], T[3])) return 422;
        if (p->high_order) {   /* low_collision_old (mod_ImplicitMicro.f90:66-79) */
            double tau_o;
            maxwell(p, nv, c->u, c->v, po, T[4], T[5]);
            shakhov(p, nv, T[4], T[5], c->u, c->v, q, po, T[0], T[1]);
            for (int k = 0; k < nv; ++k) { T[4][k] = T[4][k] + T[0][k]; T[5][k] = T[5][k] + T[1][k]; }
            memcpy(T[2], T[4], sizeof(double) * nv);
            memcpy(T[3], T[5], sizeof(double) * nv);
            if (!uo_project_moments(nv, T[4], T[5], c->W + cc * 4, c->u, c->v, c->w, T[2], T[3])) return 422;
            if ((e = get_tau(p, po, &tau_o))) return e;
            for (int k = 0; k < nv; ++k) {
                c->lco_h[(size_t)cc * nv + k] = (T[4][k] - c->h[(size_t)cc * nv + k]) / tau_o;
                c->lco_b[(size_t)cc * nv + k] = (T[5][k] - c->b[(size_t)cc * nv + k]) / tau_o;
            }
        }
    }
    /* SolveMicroLUSGS with the frozen wall closure, one sweep pair */
    memset(c->dh_ghost, 0, S * sizeof(double));
    memset(c->db_ghost, 0, S * sizeof(double));
    for (int s = 0; s < p->nslab; ++s) if (!lusgs_stage(c, s, 0, dtp)) return 423;
    memcpy(c->dh_ghost, c->dh, S * sizeof(double));           /* MPIExchangeDeltaMicro */
    memcpy(c->db_ghost, c->db, S * sizeof(double));
    for (int s = 0; s < p->nslab; ++s) if (!lusgs_stage(c, s, 1, dtp)) return 423;
    /* FindAdmissibleMicroAlpha(enforce_negative_fraction=.false.) (mod_SteadyImplicit.f90:53-117) */
    double alpha = 1.0;
    double** T = scratch_t(c, 0);
    for (;;) {
        int ok = 1;
        for (int cc = 0; cc < c->nc && ok; ++cc) {
            double mm[4];
            for (int k = 0; k < nv; ++k) {
                size_t q = (size_t)cc * nv + k;
                T[0][k] = c->h[q] + alpha * c->dh[q];
                T[1][k] = c->b[q] + alpha * c->db[q];
                ok &= isfinite(T[0][k]) && isfinite(T[1][k]);
            }
            moment_conserved(nv, T[0], T[1], c->u, c->v, c->w, mm);
            ok &= uo_is_physical(mm);
        }
        if (ok) break;
        alpha = 0.5 * alpha;
        if (alpha < p->min_alpha) return 433;
    }
    for (size_t q = 0; q < S; ++q) { c->h[q] = c->h[q] + alpha * c->dh[q]; c->b[q] = c->b[q] + alpha * c->db[q]; }
    /* RecoverMacroFromKineticState + moment gate (mod_ImplicitMicro.f90:628-645, mod_SteadyImplicit.f90:451-459) */
    for (int cc = 0; cc < c->nc; ++cc) {
        double mm[4];
        moment_conserved(nv, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv, c->u, c->v, c->w, mm);
        if (!uo_is_physical(mm)) return 434;
        memcpy(c->wt + cc * 4, mm, sizeof mm);
    }
    memcpy(c->W, c->wt, sizeof(double) * c->nc * 4);
    double merr = 0.0;
    for (int cc = 0; cc < c->nc; ++cc) {
        double mm[4];
        moment_conserved(nv, c->h + (size_t)cc * nv, c->b + (size_t)cc * nv, c->u, c->v, c->w, mm);
        for (int m = 0; m < 4; ++m) merr = fmax(merr, fabs(c->W[cc * 4 + m] - mm[m]) / fmax(fabs(c->W[cc * 4 + m]), 1.0));
    }
    if (!(merr <= p->moment_tol)) return 451;
    /* CheckR5Policy (mod_R5Observe.f90:248-256): the accepted update must be a full step */
    if (alpha != 1.0 || malpha != 1.0) return 452;
    /* RescaleClosedMass (mod_ClosedCouetteMass.f90:243-313) */
    if (p->mass_rescale) {
        double t[5], m[5];
        if (!mass_statistics(c, t, m)) return 941;
        c->mass_scale = c->m0 / t[0];
        for (int q = 0; q < c->nc * 4; ++q) c->W[q] = c->mass_scale * c->W[q];
        for (size_t q = 0; q < S; ++q) { c->h[q] = c->mass_scale * c->h[q]; c->b[q] = c->mass_scale * c->b[q]; }
    }
    /* AfterR5Accepted -> EvaluateSparseState (mod_R5Observe.f90:287-320) */
    double totals[5], metrics[5];
    if (!mass_statistics(c, totals, metrics)) return 941;
    if (p->high_order) {
        if ((e = uo_s2_evolution(c, dt))) return e;
        if ((e = uo_s2_compute_residual(c, dt, 0))) return e;
        if ((e = uo_s2_compute_residual(c, dt, 1))) return e;
    } else {
        uo_interpolation(c);
        if ((e = uo_evolution(c, dt))) return e;
        if ((e = uo_compute_residual(c, dt, 1))) return e;
        if (!reassemble_rates(c, dt)) return 444;
    }
    double sci[22];
    implicit_diagnostics(c, dt, sci);
    sci[18] = merr;   /* implicit_moment_error of this step (or the rescaled state's, below) */
    if (p->mass_rescale) sci[18] = metrics[0];
    /* flux_1..16: boundary-face totals per unit time (mod_R5Observe.f90:107-113) */
    double fl[16] = {0};
    int nx = p->nx, ny = p->ny;
    for (int j = 0; j < ny; ++j)
        for (int m = 0; m < 4; ++m) {
            fl[m] = fl[m] - c->fxw[((size_t)j * nx + 0) * 4 + m] / dt;
            fl[4 + m] = fl[4 + m] + c->fxw[((size_t)j * nx + 0) * 4 + m] / dt;
        }
    for (int i = 0; i < nx; ++i)
        for (int m = 0; m < 4; ++m) {
            fl[8 + m] = fl[8 + m] - c->fyLw[(size_t)i * 4 + m] / dt;
            fl[12 + m] = fl[12 + m] + c->fyRw[((size_t)ny * nx + i) * 4 + m] / dt;
        }
    int pass = sci[0] <= p->residual_tol && sci[1] <= p->residual_tol && sci[2] <= p->residual_tol &&
               sci[3] <= p->residual_tol && sci[12] <= p->residual_tol && sci[13] <= p->residual_tol &&
               metrics[0] <= p->moment_tol;
    c->streak = pass ? c->streak + 1 : 0;
    row[0] = pass; row[1] = metrics[0]; row[2] = totals[0]; row[3] = totals[4];
    row[4] = sci[8]; row[5] = sci[9]; row[6] = sci[10]; row[7] = sci[11];
    row[8] = sci[20]; row[9] = sci[21]; row[10] = sci[16]; row[11] = sci[17];
    memcpy(row + 12, sci, sizeof sci);
    memcpy(row + 34, fl, sizeof fl);
    row[50] = c->ref_h; row[51] = c->ref_b;
    row[52] = p->mass_rescale ? c->mass_scale - 1.0 : 0.0;
    row[53] = alpha; row[54] = malpha; row[55] = dt; row[56] = c->streak;
    if (out) memcpy(out, row, sizeof(double) * (nout < 80 ? nout : 80));
    return 0;
}

#include "ugks_oracle_s2.c"
