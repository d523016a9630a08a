// ugks_lo.cu -- second-order UGKS hot path for one Couette domain on sm_100a (FP64).
//
//   k_lo_faces  : Interpolation (mod_Interpolation.f90:26-170) fused into the face flux of
//                 EvolutionNative (mod_Evolution.f90:46-177): one CTA per face, the upwind cell's
//                 Van-Leer slopes recomputed on the fly from the L2-resident state;
//                 CalcFlux_MultiDimension (:186-492) for interior faces, W2BMultiscaleFluxBoundary
//                 (:1888-2449) for the 2*nx wall faces.
//   k_lo_cells  : ComputeResidual (mod_Residual.f90:17-132) + ApplyExplicitUpdate
//                 (mod_TimeIntegrator.f90:16-293) fused, one CTA per cell, plus the next TimeStep
//                 (mod_Solve.f90:373-421) and the residual norms reduced by the last CTA.
//
// Layout: h, b are [cell][velocity] (velocity fastest, coalesced FP64 rows); one CTA covers a
// whole velocity row with kVPT velocities per thread, so every moment sum is one block reduction.
#include "ugks_lo.cuh"

namespace ugks {

__device__ __forceinline__ int wrapx(int i, int nx) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); }

// Slope of array A at cell (i,j) in direction d for velocity k (Interp_VanLeer / InterpBoundary).
// Wall rows use the one-sided (right-left)/dy slope (mod_Interpolation.f90:40-45,78-88).
__device__ __forceinline__ double lo_slope(const LoParams& P, const double* __restrict__ A, int d, int i, int j,
                                           int k) {
    const int nv = P.nvel;
    const double a0 = A[(size_t)(j * P.nx + i) * nv + k];
    if (d == 0) {
        const double am = A[(size_t)(j * P.nx + wrapx(i - 1, P.nx)) * nv + k];
        const double ap = A[(size_t)(j * P.nx + wrapx(i + 1, P.nx)) * nv + k];
        return vanleer((a0 - am) / P.dx, (ap - a0) / P.dx);
    }
    if (j == 0) {
        const double ap = A[(size_t)((j + 1) * P.nx + i) * nv + k];
        return (ap - a0) / P.dy;
    }
    if (j == P.ny - 1) {
        const double am = A[(size_t)((j - 1) * P.nx + i) * nv + k];
        return (a0 - am) / P.dy;
    }
    const double am = A[(size_t)((j - 1) * P.nx + i) * nv + k];
    const double ap = A[(size_t)((j + 1) * P.nx + i) * nv + k];
    return vanleer((a0 - am) / P.dy, (ap - a0) / P.dy);
}

// -------------------------------------------------------------------------------------------
// Interior face: CalcFlux_MultiDimension (mod_Evolution.f90:186-492), UnifiedPhysicalOperators.
// dir 0: vertical face (vn = u, vt = v); dir 1: horizontal face (vn = v, vt = -u).
template <int VPT>
__device__ void lo_face_interior(const LoParams& P, const LoBuffers& B, int dir, int iL, int jL, int iR, int jR,
                                 double dt, double* __restrict__ Fh, double* __restrict__ Fb, double* Fw,
                                 double* red, double* rout) {
    const int nv = P.nvel, tid = threadIdx.x, NT = blockDim.x;
    const double len = dir == 0 ? P.dx : P.dy;      // cell length normal to the face
    const double flen = dir == 0 ? P.dy : P.dx;     // face length
    const double hl = 0.5 * len;
    double hv[VPT], bv[VPT], shn[VPT], sbn[VPT], sht[VPT], sbt[VPT], H0[VPT], B0[VPT];
    double acc[16];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        hv[r] = bv[r] = shn[r] = sbn[r] = sht[r] = sbt[r] = 0.0;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const bool left = copysign(1.0, vn) > 0.0;       // delta = (sign(1,vn)+1)/2
        const int ci = left ? iL : iR, cj = left ? jL : jR;
        const size_t ck = (size_t)(cj * P.nx + ci) * nv + k;
        const double sgn = left ? 1.0 : -1.0;
        const double snh = lo_slope(P, B.h, dir, ci, cj, k), snb = lo_slope(P, B.b, dir, ci, cj, k);
        const double sth = lo_slope(P, B.h, 1 - dir, ci, cj, k), stb = lo_slope(P, B.b, 1 - dir, ci, cj, k);
        hv[r] = B.h[ck] + sgn * (hl * snh);
        bv[r] = B.b[ck] + sgn * (hl * snb);
        shn[r] = snh; sbn[r] = snb;
        sht[r] = dir == 0 ? sth : -sth;
        sbt[r] = dir == 0 ? stb : -stb;
        const double v2 = vn * vn + vt * vt;
        acc[0] += wk * hv[r];
        acc[1] += wk * vn * hv[r];
        acc[2] += wk * vt * hv[r];
        acc[3] += 0.5 * wk * (v2 * hv[r] + bv[r]);
        acc[4] += wk * sht[r];
        acc[5] += wk * vn * sht[r];
        acc[6] += wk * vt * sht[r];
        acc[7] += 0.5 * wk * (v2 * sht[r] + sbt[r]);
    }
    block_reduce<8, 0>(acc, red, rout);
    // face state, slopes, collision time (every thread, identical values)
    Prim pf;
    const double cv[4] = {acc[0], acc[1], acc[2], acc[3]};
    bool ok = get_primary(P.gm1, cv, pf);
    const double* WL = B.W + (jL * P.nx + iL) * 4;
    const double* WR = B.W + (jR * P.nx + iR) * 4;
    double wl[4], wr[4];
    if (dir == 0) { wl[0] = WL[0]; wl[1] = WL[1]; wl[2] = WL[2]; wl[3] = WL[3];
                    wr[0] = WR[0]; wr[1] = WR[1]; wr[2] = WR[2]; wr[3] = WR[3]; }
    else { wl[0] = WL[0]; wl[1] = WL[2]; wl[2] = -WL[1]; wl[3] = WL[3];
           wr[0] = WR[0]; wr[1] = WR[2]; wr[2] = -WR[1]; wr[3] = WR[3]; }
    double sw[4], aL[4], aR[4], bs[4], aT[4], Mt[5], tau = 1.0;
    if (!ok) { pf.r = 1.0; pf.U = 0.0; pf.V = 0.0; pf.L = 1.0; }
#pragma unroll
    for (int m = 0; m < 4; ++m) sw[m] = (cv[m] - wl[m]) / hl;
    micro_slope(P.ck, pf, sw, aL);
#pragma unroll
    for (int m = 0; m < 4; ++m) sw[m] = (wr[m] - cv[m]) / hl;
    micro_slope(P.ck, pf, sw, aR);
    const double swt[4] = {acc[4], acc[5], acc[6], acc[7]};
    micro_slope(P.ck, pf, swt, bs);
    Moments M;
    calc_moment(P.ck, pf, M);
    {
        double MauL[4], MauR[4], Mbv[4];
        moment_auvxi(aL, M.MuL, M.Mv, M.Mxi, 1, 0, MauL);
        moment_auvxi(aR, M.MuR, M.Mv, M.Mxi, 1, 0, MauR);
        moment_auvxi(bs, M.Mu, M.Mv, M.Mxi, 0, 1, Mbv);
#pragma unroll
        for (int m = 0; m < 4; ++m) sw[m] = -pf.r * (MauL[m] + MauR[m] + Mbv[m]);
        micro_slope(P.ck, pf, sw, aT);
    }
    const bool tok = get_tau(P.mu_ref, P.omega, pf, tau);
    if (!tok) tau = 1.0;
    time_coeffs(dt, tau, Mt);
    if (tid == 0) {
        if (!ok) set_status(B.status, ST_GETPRIMARY);
        if (ok && !tok) set_status(B.status, ST_TAU);
    }
    // face equilibrium H0, B0 (PrepareNativeFaceEquilibrium, mod_Evolution.f90:16-30) + heat flux
    const double pref = pf.r * (pf.L / kPi), bfac = (double)P.ck / (2.0 * pf.L);
    acc[0] = acc[1] = 0.0;
    acc[2] = acc[3] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        H0[r] = B0[r] = 0.0;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const double dvn = vn - pf.U, dvt = vt - pf.V, v2 = dvn * dvn + dvt * dvt;
        H0[r] = pref * exp(-pf.L * v2);
        B0[r] = H0[r] * bfac;
        acc[0] += 0.5 * wk * dvn * (v2 * hv[r] + bv[r]);
        acc[1] += 0.5 * wk * dvt * (v2 * hv[r] + bv[r]);
        acc[2] = fmax(acc[2], fabs(H0[r]));
        acc[3] = fmax(acc[3], fabs(B0[r]));
    }
    block_reduce<2, 2>(acc, red, rout);
    const double qf0 = acc[0], qf1 = acc[1];
    const double sch = fmax(acc[2], 1.0), scb = fmax(acc[3], 1.0);
    // ProjectToConservedMoments of H0,B0 onto GetConserved(pf) in the local frame
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        moment_add(wk, vn, vt, H0[r], B0[r], acc);
        gram_add(wk, fmax(fabs(H0[r]), kEps * sch), fmax(fabs(B0[r]), kEps * scb), vn, vt, acc + 4);
    }
    block_reduce<14, 0>(acc, red, rout);
    double tgt[4], rhs[4], gm[16], lam[4];
    get_conserved(P.gm1, pf, tgt);
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = tgt[m] - acc[m];
    gram_expand(acc + 4, gm);
    const bool pok = solve_dense4(gm, rhs, lam);
    if (!pok) { lam[0] = lam[1] = lam[2] = lam[3] = 0.0; }
    // Shakhov part and the micro flux (mod_Evolution.f90:396-453), scaled by the face length.
    const double coeff = 0.8 * (1.0 - P.pr) * pf.L * pf.L / pf.r;
    const double c2ck = 2.0 / (double)P.ck;
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double a = dir == 0 ? uk : vk, t = dir == 0 ? vk : -uk;
        const double wh = fmax(fabs(H0[r]), kEps * sch), wb = fmax(fabs(B0[r]), kEps * scb);
        const double e = 0.5 * (a * a + t * t);
        const double H = H0[r] + wh * (lam[0] + a * lam[1] + t * lam[2] + e * lam[3]);
        const double Bq = B0[r] + 0.5 * wb * lam[3];
        moment_add(wk, a, t, H, Bq, acc);   // projection gate
        const double dvn = a - pf.U, dvt = t - pf.V, dv2 = dvn * dvn + dvt * dvt;
        const double qdot = dvn * qf0 + dvt * qf1;
        const double shH = 2.0 * pf.L * dv2 - 4.0, shB = shH + c2ck;
        const double Hp = coeff * qdot * shH * H, Bp = coeff * qdot * shB * Bq;
        const double v2 = a * a + t * t;
        const bool left = copysign(1.0, a) > 0.0;
        const double slh = a * shn[r] + t * sht[r], slb = a * sbn[r] + t * sbt[r];
        const double* as = left ? aL : aR;
        const double h_a = as[0] * H + as[1] * a * H + as[2] * t * H + 0.5 * as[3] * (v2 * H + Bq);
        const double h_b = bs[0] * H + bs[1] * a * H + bs[2] * t * H + 0.5 * bs[3] * (v2 * H + Bq);
        const double h_T = aT[0] * H + aT[1] * a * H + aT[2] * t * H + 0.5 * aT[3] * (v2 * H + Bq);
        const double b_a = as[0] * Bq + as[1] * a * Bq + as[2] * t * Bq + 0.5 * as[3] * (v2 * Bq + M.Mxi[2] * H);
        const double b_b = bs[0] * Bq + bs[1] * a * Bq + bs[2] * t * Bq + 0.5 * bs[3] * (v2 * Bq + M.Mxi[2] * H);
        const double b_T = aT[0] * Bq + aT[1] * a * Bq + aT[2] * t * Bq + 0.5 * aT[3] * (v2 * Bq + M.Mxi[2] * H);
        const double fh = Mt[0] * a * (H + Hp) + Mt[1] * a * a * h_a + Mt[1] * a * t * h_b + Mt[2] * a * h_T +
                          Mt[3] * a * hv[r] - Mt[4] * a * slh;
        const double fb = Mt[0] * a * (Bq + Bp) + Mt[1] * a * a * b_a + Mt[1] * a * t * b_b + Mt[2] * a * b_T +
                          Mt[3] * a * bv[r] - Mt[4] * a * slb;
        const double Fhk = flen * fh, Fbk = flen * fb;
        Fh[k] = Fhk;
        Fb[k] = Fbk;
        moment_add(wk, uk, vk, Fhk, Fbk, acc + 4);   // MomentConserved in the global frame (:470-473)
    }
    block_reduce<8, 0>(acc, red, rout);
    if (tid == 0) {
        const double rs = fmax(fmax(fmax(fabs(tgt[0]), fabs(tgt[1])), fmax(fabs(tgt[2]), fabs(tgt[3]))), 1.0);
        double err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) err = fmax(err, fabs(acc[m] - tgt[m]));
        if (!pok || !(err <= 1.0e-10 * rs)) set_status(B.status, ST_FACE_PROJECTION);
        bool fin = true;
#pragma unroll
        for (int m = 0; m < 4; ++m) { Fw[m] = acc[4 + m]; fin = fin && isfinite(acc[4 + m]); }
        if (!fin) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// -------------------------------------------------------------------------------------------
// Wall face: W2BMultiscaleFluxBoundary (mod_Evolution.f90:1888-2449) on the horizontal walls.
// side -1: bottom wall below row 0 (Lside); +1: top wall above row ny-1 (Rside).
template <int VPT>
__device__ void lo_face_wall(const LoParams& P, const LoBuffers& B, int side, int i, double dt,
                             double* __restrict__ Fh, double* __restrict__ Fb, double* Fw, double* aero,
                             double* red, double* rout) {
    const int nv = P.nvel, tid = threadIdx.x, NT = blockDim.x;
    const int iw = side < 0 ? 0 : 1;
    const int j = side < 0 ? 0 : P.ny - 1;
    const int cell = j * P.nx + i;
    const double len = P.dy, flen = P.dx;
    const double rot = -(double)side;
    double hv[VPT], bv[VPT], shn[VPT], sbn[VPT], sht[VPT], sbt[VPT], Hg[VPT], Bg[VPT], Hw[VPT], Bw[VPT];
    // wall and cell states in the local frame (vn = v, vt = -u)
    const double* Wc = B.W + cell * 4;
    Prim pc;
    const bool ok = get_primary(P.gm1, Wc, pc);
    Prim prim{pc.r, pc.V, -pc.U, pc.L};
    Prim pw{1.0, P.wall_ux[iw] * (-0.0) + 0.0 * 1.0, -P.wall_ux[iw] * 1.0 + 0.0 * (-0.0), P.wall_lam[iw]};
    Prim pg = pw;
    pg.r = prim.r / prim.L * pw.L;
    double tau = 1.0, Mt[5];
    const bool tok = get_tau(P.mu_ref, P.omega, pg, tau);
    if (!tok) tau = 1.0;
    time_coeffs(dt, tau, Mt);
    if (tid == 0) {
        if (!ok) set_status(B.status, ST_GETPRIMARY);
        if (ok && !tok) set_status(B.status, ST_TAU);
    }
    const double prefg = pg.r * (pg.L / kPi), prefw = 1.0 * (pw.L / kPi), bfac = (double)P.ck / (2.0 * pw.L);
    double acc[40];
#pragma unroll
    for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        hv[r] = bv[r] = shn[r] = sbn[r] = sht[r] = sbt[r] = Hg[r] = Bg[r] = Hw[r] = Bw[r] = 0.0;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double vn = vk, vt = -uk;
        const size_t ckk = (size_t)cell * nv + k;
        shn[r] = lo_slope(P, B.h, 1, i, j, k);
        sbn[r] = lo_slope(P, B.b, 1, i, j, k);
        sht[r] = -lo_slope(P, B.h, 0, i, j, k);
        sbt[r] = -lo_slope(P, B.b, 0, i, j, k);
        hv[r] = B.h[ckk] - rot * 0.5 * len * shn[r];
        bv[r] = B.b[ckk] - rot * 0.5 * len * sbn[r];
        const double dvn = vn - pg.U, dvt = vt - pg.V, v2 = dvn * dvn + dvt * dvt;
        const double ex = exp(-pg.L * v2);
        Hg[r] = prefg * ex;
        Bg[r] = Hg[r] * bfac;
        Hw[r] = prefw * ex;
        Bw[r] = Hw[r] * bfac;
        const double lv2 = vn * vn + vt * vt;
        acc[0] += wk * sht[r];
        acc[1] += wk * vn * sht[r];
        acc[2] += wk * vt * sht[r];
        acc[3] += 0.5 * wk * (lv2 * sht[r] + sbt[r]);
        acc[4] += 0.5 * wk * dvn * (v2 * hv[r] + bv[r]);
        acc[5] += 0.5 * wk * dvt * (v2 * hv[r] + bv[r]);
        acc[6] = fmax(acc[6], fabs(Hg[r]));
        acc[7] = fmax(acc[7], fabs(Bg[r]));
        acc[8] = fmax(acc[8], fabs(Hw[r]));
        acc[9] = fmax(acc[9], fabs(Bw[r]));
    }
    block_reduce<6, 4>(acc, red, rout);
    const double swt[4] = {acc[0], acc[1], acc[2], acc[3]};
    const double qf0 = acc[4], qf1 = acc[5];
    const double sgh = fmax(acc[6], 1.0), sgb = fmax(acc[7], 1.0), swh = fmax(acc[8], 1.0), swb = fmax(acc[9], 1.0);
    // micro slopes a_gn, a_gt, a_T (mod_Evolution.f90:2044-2087)
    double cg[4], a_gn[4], a_gt[4], a_T[4], sw[4];
    get_conserved(P.gm1, pg, cg);
    const double cg1[4] = {Wc[0], Wc[2], -Wc[1], Wc[3]};
#pragma unroll
    for (int m = 0; m < 4; ++m) sw[m] = (cg[m] - cg1[m]) / ((double)side * 0.5 * len);
    micro_slope(P.ck, pg, sw, a_gn);
    micro_slope(P.ck, pg, swt, a_gt);
    Moments M;
    calc_moment(P.ck, pg, M);
    {
        double Mau[4], Mbv[4];
        moment_auvxi(a_gn, M.Mu, M.Mv, M.Mxi, 1, 0, Mau);
        moment_auvxi(a_gt, M.Mu, M.Mv, M.Mxi, 0, 1, Mbv);
#pragma unroll
        for (int m = 0; m < 4; ++m) sw[m] = -pg.r * (Mau[m] + Mbv[m]);
        micro_slope(P.ck, pg, sw, a_T);
    }
    // two face-equilibrium projections (H_g onto GetConserved(pg), H_w onto GetConserved(pshape))
#pragma unroll
    for (int m = 0; m < 28; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double vn = vk, vt = -uk;
        moment_add(wk, vn, vt, Hg[r], Bg[r], acc);
        gram_add(wk, fmax(fabs(Hg[r]), kEps * sgh), fmax(fabs(Bg[r]), kEps * sgb), vn, vt, acc + 4);
        moment_add(wk, vn, vt, Hw[r], Bw[r], acc + 14);
        gram_add(wk, fmax(fabs(Hw[r]), kEps * swh), fmax(fabs(Bw[r]), kEps * swb), vn, vt, acc + 18);
    }
    block_reduce<28, 0>(acc, red, rout);
    double tg[4], tw[4], rhs[4], gm[16], lg[4], lw[4];
    const Prim pshape{1.0, pw.U, pw.V, pw.L};
    get_conserved(P.gm1, pg, tg);
    get_conserved(P.gm1, pshape, tw);
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = tg[m] - acc[m];
    gram_expand(acc + 4, gm);
    bool pok = solve_dense4(gm, rhs, lg);
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = tw[m] - acc[14 + m];
    gram_expand(acc + 18, gm);
    pok = solve_dense4(gm, rhs, lw) && pok;
    if (!pok) { lg[0] = lg[1] = lg[2] = lg[3] = lw[0] = lw[1] = lw[2] = lw[3] = 0.0; }
    const double coeff = 0.8 * (1.0 - P.pr) * pg.L * pg.L / pg.r;
    const double c2ck = 2.0 / (double)P.ck;
#pragma unroll
    for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double a = vk, t = -uk, e = 0.5 * (a * a + t * t);
        Hg[r] = Hg[r] + fmax(fabs(Hg[r]), kEps * sgh) * (lg[0] + a * lg[1] + t * lg[2] + e * lg[3]);
        Bg[r] = Bg[r] + 0.5 * fmax(fabs(Bg[r]), kEps * sgb) * lg[3];
        Hw[r] = Hw[r] + fmax(fabs(Hw[r]), kEps * swh) * (lw[0] + a * lw[1] + t * lw[2] + e * lw[3]);
        Bw[r] = Bw[r] + 0.5 * fmax(fabs(Bw[r]), kEps * swb) * lw[3];
        moment_add(wk, a, t, Hg[r], Bg[r], acc + 2);
        moment_add(wk, a, t, Hw[r], Bw[r], acc + 6);
        const double dk = (copysign(1.0, a) * rot + 1.0) / 2.0, ik = 1.0 - dk;
        const double slh = a * shn[r] + t * sht[r];
        const double v2 = a * a + t * t;
        const double dvn = a - pg.U, dvt = t - pg.V, dv2 = dvn * dvn + dvt * dvt;
        const double Hp = coeff * (dvn * qf0 + dvt * qf1) * (2.0 * pg.L * dv2 - 4.0) * Hg[r];
        const double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hg[r] + 0.5 * a_gn[3] * (v2 * Hg[r] + Bg[r]);
        const double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hg[r] + 0.5 * a_gt[3] * (v2 * Hg[r] + Bg[r]);
        const double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hg[r] + 0.5 * a_T[3] * (v2 * Hg[r] + Bg[r]);
        acc[0] += wk * a * ik * (Mt[0] * (Hg[r] + Hp) + Mt[1] * (a * Ha_gn + t * Ha_gt) + Mt[2] * Ha_T +
                                 Mt[3] * hv[r] - Mt[4] * slh);
        acc[1] += wk * a * Hw[r] * dk;
        (void)c2ck;
    }
    block_reduce<10, 0>(acc, red, rout);
    const double rhow = -acc[0] / (dt * acc[1]);   // prim_w(1) = -incidence/reflection
    if (tid == 0) {
        const double rg = fmax(fmax(fmax(fabs(tg[0]), fabs(tg[1])), fmax(fabs(tg[2]), fabs(tg[3]))), 1.0);
        const double rw = fmax(fmax(fmax(fabs(tw[0]), fabs(tw[1])), fmax(fabs(tw[2]), fabs(tw[3]))), 1.0);
        double eg = 0.0, ew = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { eg = fmax(eg, fabs(acc[2 + m] - tg[m])); ew = fmax(ew, fabs(acc[6 + m] - tw[m])); }
        if (!pok || !(eg <= 1.0e-10 * rg) || !(ew <= 1.0e-10 * rw)) set_status(B.status, ST_FACE_PROJECTION);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        const double a = vk, t = -uk, v2 = a * a + t * t;
        const double dk = (copysign(1.0, a) * rot + 1.0) / 2.0, ik = 1.0 - dk;
        const double Hwk = rhow * Hw[r], Bwk = rhow * Bw[r];
        const double Hgk = Hg[r], Bgk = Bg[r];
        const double dvn = a - pg.U, dvt = t - pg.V, dv2 = dvn * dvn + dvt * dvt;
        const double qdot = dvn * qf0 + dvt * qf1;
        const double shH = 2.0 * pg.L * dv2 - 4.0;
        const double Hp = coeff * qdot * shH * Hgk, Bp = coeff * qdot * (shH + c2ck) * Bgk;
        const double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hgk + 0.5 * a_gn[3] * (v2 * Hgk + Bgk);
        const double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hgk + 0.5 * a_gt[3] * (v2 * Hgk + Bgk);
        const double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hgk + 0.5 * a_T[3] * (v2 * Hgk + Bgk);
        const double Ba_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Bgk + 0.5 * a_gn[3] * (v2 * Bgk + M.Mxi[2] * Hgk);
        const double Ba_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Bgk + 0.5 * a_gt[3] * (v2 * Bgk + M.Mxi[2] * Hgk);
        const double Ba_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Bgk + 0.5 * a_T[3] * (v2 * Bgk + M.Mxi[2] * Hgk);
        const double fh = flen * (dt * a * Hwk * dk + Mt[0] * a * (Hgk + Hp) * ik + Mt[1] * a * a * Ha_gn * ik +
                                  Mt[1] * a * t * Ha_gt * ik + Mt[2] * a * Ha_T * ik + Mt[3] * a * hv[r] * ik -
                                  Mt[4] * a * (a * shn[r] + t * sht[r]) * ik);
        const double fb = flen * (dt * a * Bwk * dk + Mt[0] * a * (Bgk + Bp) * ik + Mt[1] * a * a * Ba_gn * ik +
                                  Mt[1] * a * t * Ba_gt * ik + Mt[2] * a * Ba_T * ik + Mt[3] * a * bv[r] * ik -
                                  Mt[4] * a * (a * sbn[r] + t * sbt[r]) * ik);
        Fh[k] = fh;
        Fb[k] = fb;
        const double hk = fh / flen, bk = fb / flen;
        acc[0] += wk * hk;
        acc[1] += wk * (a * hk);
        acc[2] += wk * (t * hk);
        acc[3] += wk * (0.5 * (v2 * hk + bk));
    }
    block_reduce<4, 0>(acc, red, rout);
    if (tid == 0) {
        aero[0] = acc[1] / dt;
        aero[1] = acc[2] / dt;
        aero[2] = acc[3] / dt - pw.V * acc[2] / dt;
        // GlobalFrame with cosx = -0, cosy = 1: [f1, -f3, f2, f4], then times the face length
        Fw[0] = flen * acc[0];
        Fw[1] = flen * (-acc[2]);
        Fw[2] = flen * acc[1];
        Fw[3] = flen * acc[3];
        if (!(isfinite(acc[0]) && isfinite(acc[1]) && isfinite(acc[2]) && isfinite(acc[3])))
            set_status(B.status, ST_NONFINITE_FLUX);
    }
}

template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX) k_lo_faces(LoParams P, LoBuffers B) {
    __shared__ double red[32 * kRedSlots];
    __shared__ double rout[kRedSlots];
    const double dt = B.dt[0];
    const int nx = P.nx, ny = P.ny, nv = P.nvel;
    int f = blockIdx.x;
    if (f < nx * ny) {
        const int j = f / nx, i = f % nx;
        const size_t o = (size_t)(j * nx + i);
        lo_face_interior<VPT>(P, B, 0, wrapx(i - 1, nx), j, i, j, dt, B.fxh + o * nv, B.fxb + o * nv, B.fxw + o * 4,
                              red, rout);
        return;
    }
    f -= nx * ny;
    if (f < nx * (ny - 1)) {
        const int jf = 1 + f / nx, i = f % nx;
        const size_t o = (size_t)(jf * nx + i);
        lo_face_interior<VPT>(P, B, 1, i, jf - 1, i, jf, dt, B.fyh + o * nv, B.fyb + o * nv, B.fyw + o * 4, red,
                              rout);
        return;
    }
    f -= nx * (ny - 1);
    const int side = f < nx ? -1 : 1, i = f % nx;
    const size_t o = (size_t)((side < 0 ? 0 : ny) * nx + i);
    lo_face_wall<VPT>(P, B, side, i, dt, B.fyh + o * nv, B.fyb + o * nv, B.fyw + o * 4,
                      B.wall_aero + ((side < 0 ? 0 : 1) * nx + i) * 3, red, rout);
}

// -------------------------------------------------------------------------------------------
// Per-cell TimeStep (mod_Solve.f90:386-405): dt_local = CFL*area/(dy*max(U_MAX,|U|+c)+dx*max(V_MAX,|V|+c))
__device__ __forceinline__ double cell_dt(const LoParams& P, const double w[4], bool& ok) {
    Prim p;
    ok = get_primary(P.gm1, w, p);
    if (!ok) return 0.0;
    const double sos = sqrt(0.5 * (P.gm1 + 1.0) / p.L);
    const double a = fmax(P.umax, fabs(p.U) + sos), bq = fmax(P.vmax, fabs(p.V) + sos);
    return P.cfl * P.area / (P.dy * a + P.dx * bq);
}

// Last-CTA epilogue: dt_global = min(dt_local) (MPI_AllReduce MIN, mod_Solve.f90:409-418) and
// the residual-norm sums (mod_TimeIntegrator.f90:102-106), reduced in a fixed order.
__device__ void last_cta_epilogue(const LoParams& P, const LoBuffers& B, bool write_dt, bool write_diag,
                                  double* red, double* rout) {
    __shared__ unsigned s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(B.counter, 1u) == (unsigned)(gridDim.x - 1)) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nc = P.nx * P.ny;
    double acc[kNDiag + 1];
#pragma unroll
    for (int m = 0; m < kNDiag; ++m) acc[m] = 0.0;
    acc[kNDiag] = -INFINITY;   // max of -dt_local == -min(dt_local)
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        if (write_dt) acc[kNDiag] = fmax(acc[kNDiag], -__ldcg(B.dtl + c));
        if (write_diag) {
#pragma unroll
            for (int m = 0; m < 9; ++m) acc[m] += __ldcg(B.cell_diag + (size_t)c * kNDiag + m);
        }
    }
    // maxima (res_max) are reduced as sums of nothing here; do them separately below
    block_reduce<9, 0>(acc, red, rout);
    double mx[5];
    for (int m = 0; m < 4; ++m) mx[m] = 0.0;
    mx[4] = acc[kNDiag];
    for (int c = threadIdx.x; c < nc && write_diag; c += blockDim.x)
        for (int m = 0; m < 4; ++m) mx[m] = fmax(mx[m], __ldcg(B.cell_diag + (size_t)c * kNDiag + 9 + m));
    block_reduce<0, 5>(mx, red, rout);
    if (threadIdx.x == 0) {
        if (write_diag) {
            for (int m = 0; m < 9; ++m) B.diag[m] = acc[m];
            for (int m = 0; m < 4; ++m) B.diag[9 + m] = mx[m];
        }
        if (write_dt) {
            B.dt[1] = B.dt[0];   // dt_global of the step that just completed
            B.dt[0] = P.fixed_dt > 0.0 ? P.fixed_dt : -mx[4];
        }
        *B.counter = 0u;
    }
}

__global__ void __launch_bounds__(256) k_lo_timestep(LoParams P, LoBuffers B) {
    __shared__ double red[32 * kRedSlots];
    __shared__ double rout[kRedSlots];
    const int nc = P.nx * P.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        bool ok;
        const double d = cell_dt(P, B.W + c * 4, ok);
        B.dtl[c] = d;
        if (!ok) set_status(B.status, ST_GETPRIMARY);
    }
    last_cta_epilogue(P, B, true, false, red, rout);
}

// -------------------------------------------------------------------------------------------
// Cell kernel.  MODE_RESIDUAL: ComputeResidual only (res_w, res_h, res_b and, with collision,
// the physical equilibrium/collision of AssembleSteadyRateResiduals).  MODE_UPDATE: reads the
// cached residual and applies ApplyExplicitUpdate.  MODE_FUSED: both, no residual round trip.
enum { MODE_RESIDUAL = 1, MODE_UPDATE = 2, MODE_FUSED = 3 };

template <int VPT, int NTMAX, int MODE, bool COLLISION>
__global__ void __launch_bounds__(NTMAX) k_lo_cells(LoParams P, LoBuffers B) {
    __shared__ double red[32 * kRedSlots];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, tid = threadIdx.x, NT = blockDim.x, nx = P.nx;
    const int c = blockIdx.x, i = c % nx, j = c / nx;
    const double dt = B.dt[0];
    const double* hc = B.h + (size_t)c * nv;
    const double* bc = B.b + (size_t)c * nv;
    double h[VPT], b[VPT], rh[VPT], rb[VPT];
    double Wold[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) Wold[m] = B.W[c * 4 + m];
    double resw[4];
    double acc[40];
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        h[r] = b[r] = rh[r] = rb[r] = 0.0;
        if (k < nv) { h[r] = hc[k]; b[r] = bc[k]; }
    }
    if (MODE & MODE_RESIDUAL) {
        // AssembleMacroResidual / AssembleMicroFluxResidual (mod_Residual.f90:30-76)
        const size_t fl = (size_t)(j * nx + i), fr = (size_t)(j * nx + wrapx(i + 1, nx));
        const size_t gl = (size_t)(j * nx + i), gr = (size_t)((j + 1) * nx + i);
        const double area_inv = 1.0 / P.area;
#pragma unroll
        for (int m = 0; m < 4; ++m)
            resw[m] = (B.fxw[fl * 4 + m] - B.fxw[fr * 4 + m] + B.fyw[gl * 4 + m] - B.fyw[gr * 4 + m]) / P.area;
        const double dti = 1.0 / dt;
#pragma unroll
        for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            const double sh = (B.fxh[fl * nv + k] - B.fxh[fr * nv + k] + B.fyh[gl * nv + k] - B.fyh[gr * nv + k]) * area_inv;
            const double sb = (B.fxb[fl * nv + k] - B.fxb[fr * nv + k] + B.fyb[gl * nv + k] - B.fyb[gr * nv + k]) * area_inv;
            rh[r] = sh * dti;   // stream_h
            rb[r] = sb * dti;
            moment_add(B.w[k], B.u[k], B.v[k], rh[r], rb[r], acc);
            acc[4] = fmax(acc[4], fabs(h[r]));
            acc[5] = fmax(acc[5], fabs(b[r]));
        }
        block_reduce<4, 2>(acc, red, rout);
        // EnforceStreamingMomentCompatibility (mod_ImplicitMicro.f90:293-306): stream onto rate_w
        double rate[4], rhs[4], gm[16], lam[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) { rate[m] = resw[m] * dti; rhs[m] = rate[m] - acc[m]; }
        const double sh_ = fmax(acc[4], 1.0), sb_ = fmax(acc[5], 1.0);
#pragma unroll
        for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            gram_add(B.w[k], fmax(fabs(h[r]), kEps * sh_), fmax(fabs(b[r]), kEps * sb_), B.u[k], B.v[k], acc);
        }
        block_reduce<10, 0>(acc, red, rout);
        gram_expand(acc, gm);
        bool pok = solve_dense4(gm, rhs, lam);
        if (!pok) lam[0] = lam[1] = lam[2] = lam[3] = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            const double uk = B.u[k], vk = B.v[k];
            const double e = 0.5 * (uk * uk + vk * vk);
            rh[r] = rh[r] + fmax(fabs(h[r]), kEps * sh_) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
            rb[r] = rb[r] + 0.5 * fmax(fabs(b[r]), kEps * sb_) * lam[3];
            moment_add(B.w[k], uk, vk, rh[r], rb[r], acc);
            rh[r] = rh[r] * dt;   // res_h_flux_store = stream_h * dt (mod_Residual.f90:114-115)
            rb[r] = rb[r] * dt;
        }
        block_reduce<4, 0>(acc, red, rout);
        if (tid == 0) {
            const double rs = fmax(fmax(fmax(fabs(rate[0]), fabs(rate[1])), fmax(fabs(rate[2]), fabs(rate[3]))), 1.0);
            double err = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) err = fmax(err, fabs(acc[m] - rate[m]));
            if (!pok || !(err <= 1.0e-10 * rs)) set_status(B.status, ST_PROJECTION);
        }
        if (MODE == MODE_RESIDUAL) {
#pragma unroll
            for (int r = 0; r < VPT; ++r) {
                const int k = tid + r * NT;
                if (k >= nv) continue;
                B.res_h[(size_t)c * nv + k] = rh[r];
                B.res_b[(size_t)c * nv + k] = rb[r];
            }
            if (tid < 4) B.res_w[c * 4 + tid] = resw[tid];
        }
    } else {
#pragma unroll
        for (int m = 0; m < 4; ++m) resw[m] = B.res_w[c * 4 + m];
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k < nv) { rh[r] = B.res_h[(size_t)c * nv + k]; rb[r] = B.res_b[(size_t)c * nv + k]; }
        }
    }

    if (MODE == MODE_RESIDUAL && COLLISION) {
        // physical equilibrium and collision (mod_Residual.f90:116-127)
        Prim p;
        double tau = 1.0;
        const bool ok = get_primary(P.gm1, Wold, p);
        const bool tok = ok && get_tau(P.mu_ref, P.omega, p, tau);
        if (!ok) { p.r = 1.0; p.U = p.V = 0.0; p.L = 1.0; }
        if (!tok) tau = 1.0;
        if (tid == 0 && !(ok && tok)) set_status(B.status, ok ? ST_TAU : ST_GETPRIMARY);
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            const double dvn = B.u[k] - p.U, dvt = B.v[k] - p.V, v2 = dvn * dvn + dvt * dvt;
            acc[0] += 0.5 * B.w[k] * dvn * (v2 * h[r] + b[r]);
            acc[1] += 0.5 * B.w[k] * dvt * (v2 * h[r] + b[r]);
        }
        block_reduce<2, 0>(acc, red, rout);
        const double q0 = acc[0], q1 = acc[1];
        double E[VPT], F[VPT];
        const double pref = p.r * (p.L / kPi), bfac = (double)P.ck / (2.0 * p.L);
        const double coeff = 0.8 * (1.0 - P.pr) * p.L * p.L / p.r, c2ck = 2.0 / (double)P.ck;
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            E[r] = F[r] = 0.0;
            if (k >= nv) continue;
            const double dvn = B.u[k] - p.U, dvt = B.v[k] - p.V, v2 = dvn * dvn + dvt * dvt;
            const double H = pref * exp(-p.L * v2), Bm = H * bfac;
            const double qd = dvn * q0 + dvt * q1, sH = 2.0 * p.L * v2 - 4.0;
            E[r] = H + coeff * qd * sH * H;
            F[r] = Bm + coeff * qd * (sH + c2ck) * Bm;
            acc[0] = fmax(acc[0], fabs(E[r]));
            acc[1] = fmax(acc[1], fabs(F[r]));
        }
        block_reduce<0, 2>(acc, red, rout);
        const double se = fmax(acc[0], 1.0), sf = fmax(acc[1], 1.0);
#pragma unroll
        for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            moment_add(B.w[k], B.u[k], B.v[k], E[r], F[r], acc);
            gram_add(B.w[k], fmax(fabs(E[r]), kEps * se), fmax(fabs(F[r]), kEps * sf), B.u[k], B.v[k], acc + 4);
        }
        block_reduce<14, 0>(acc, red, rout);
        double rhs[4], gm[16], lam[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = Wold[m] - acc[m];
        gram_expand(acc + 4, gm);
        const bool pok = solve_dense4(gm, rhs, lam);
        if (!pok) lam[0] = lam[1] = lam[2] = lam[3] = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            if (k >= nv) continue;
            const double uk = B.u[k], vk = B.v[k], e = 0.5 * (uk * uk + vk * vk);
            const double Ep = E[r] + fmax(fabs(E[r]), kEps * se) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
            const double Fp = F[r] + 0.5 * fmax(fabs(F[r]), kEps * sf) * lam[3];
            moment_add(B.w[k], uk, vk, Ep, Fp, acc);
            B.peq_h[(size_t)c * nv + k] = Ep;
            B.peq_b[(size_t)c * nv + k] = Fp;
            B.pcol_h[(size_t)c * nv + k] = (Ep - h[r]) / tau;
            B.pcol_b[(size_t)c * nv + k] = (Fp - b[r]) / tau;
        }
        block_reduce<4, 0>(acc, red, rout);
        if (tid == 0) {
            const double rs = fmax(fmax(fmax(fabs(Wold[0]), fabs(Wold[1])), fmax(fabs(Wold[2]), fabs(Wold[3]))), 1.0);
            double err = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) err = fmax(err, fabs(acc[m] - Wold[m]));
            if (!pok || !(err <= 1.0e-10 * rs)) set_status(B.status, ST_PROJECTION);
        }
    }
    if (!(MODE & MODE_UPDATE)) return;

    // ---- ApplyExplicitUpdate (mod_TimeIntegrator.f90:16-134, 235-293)
    Prim po, pn;
    double to = 1.0, tn = 1.0, Wn[4];
    bool ok = get_primary(P.gm1, Wold, po);
    ok = ok && get_tau(P.mu_ref, P.omega, po, to);
#pragma unroll
    for (int m = 0; m < 4; ++m) Wn[m] = Wold[m] + resw[m];
    bool ok2 = get_primary(P.gm1, Wn, pn);
    ok2 = ok2 && get_tau(P.mu_ref, P.omega, pn, tn);
    if (!ok) { po.r = 1.0; po.U = po.V = 0.0; po.L = 1.0; to = 1.0; }
    if (!ok2) { pn.r = 1.0; pn.U = pn.V = 0.0; pn.L = 1.0; tn = 1.0; }
    if (tid == 0 && !(ok && ok2)) set_status(B.status, ST_GETPRIMARY);
    // heat flux of the old state (GetHeatFlux_Vec with prim_old)
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double dvn = B.u[k] - po.U, dvt = B.v[k] - po.V, v2 = dvn * dvn + dvt * dvt;
        acc[0] += 0.5 * B.w[k] * dvn * (v2 * h[r] + b[r]);
        acc[1] += 0.5 * B.w[k] * dvt * (v2 * h[r] + b[r]);
    }
    block_reduce<2, 0>(acc, red, rout);
    const double q0 = acc[0], q1 = acc[1];
    double Ho[VPT], Bo[VPT], Hn[VPT], Bn[VPT];
    {
        const double pro = po.r * (po.L / kPi), bfo = (double)P.ck / (2.0 * po.L);
        const double prn = pn.r * (pn.L / kPi), bfn = (double)P.ck / (2.0 * pn.L);
        const double co = 0.8 * (1.0 - P.pr) * po.L * po.L / po.r, cn = 0.8 * (1.0 - P.pr) * pn.L * pn.L / pn.r;
        const double c2ck = 2.0 / (double)P.ck;
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const int k = tid + r * NT;
            Ho[r] = Bo[r] = Hn[r] = Bn[r] = 0.0;
            if (k >= nv) continue;
            const double uk = B.u[k], vk = B.v[k];
            double dvn = uk - po.U, dvt = vk - po.V, v2 = dvn * dvn + dvt * dvt;
            double H = pro * exp(-po.L * v2), Bm = H * bfo, qd = dvn * q0 + dvt * q1, sH = 2.0 * po.L * v2 - 4.0;
            Ho[r] = H + co * qd * sH * H;
            Bo[r] = Bm + co * qd * (sH + c2ck) * Bm;
            dvn = uk - pn.U; dvt = vk - pn.V; v2 = dvn * dvn + dvt * dvt;
            H = prn * exp(-pn.L * v2); Bm = H * bfn; qd = dvn * q0 + dvt * q1; sH = 2.0 * pn.L * v2 - 4.0;
            Hn[r] = H + cn * qd * sH * H;
            Bn[r] = Bm + cn * qd * (sH + c2ck) * Bm;
            acc[0] = fmax(acc[0], fabs(Ho[r]));
            acc[1] = fmax(acc[1], fabs(Bo[r]));
            acc[2] = fmax(acc[2], fabs(Hn[r]));
            acc[3] = fmax(acc[3], fabs(Bn[r]));
        }
        block_reduce<0, 4>(acc, red, rout);
    }
    const double sHo = fmax(acc[0], 1.0), sBo = fmax(acc[1], 1.0), sHn = fmax(acc[2], 1.0), sBn = fmax(acc[3], 1.0);
#pragma unroll
    for (int m = 0; m < 28; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k];
        moment_add(wk, uk, vk, Ho[r], Bo[r], acc);
        gram_add(wk, fmax(fabs(Ho[r]), kEps * sHo), fmax(fabs(Bo[r]), kEps * sBo), uk, vk, acc + 4);
        moment_add(wk, uk, vk, Hn[r], Bn[r], acc + 14);
        gram_add(wk, fmax(fabs(Hn[r]), kEps * sHn), fmax(fabs(Bn[r]), kEps * sBn), uk, vk, acc + 18);
    }
    block_reduce<28, 0>(acc, red, rout);
    double to4[4], rhs[4], gm[16], lo[4], ln[4];
    get_conserved(P.gm1, po, to4);
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = to4[m] - acc[m];
    gram_expand(acc + 4, gm);
    bool pok = solve_dense4(gm, rhs, lo);
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = Wn[m] - acc[14 + m];
    gram_expand(acc + 18, gm);
    pok = solve_dense4(gm, rhs, ln) && pok;
    if (!pok) lo[0] = lo[1] = lo[2] = lo[3] = ln[0] = ln[1] = ln[2] = ln[3] = 0.0;
    const double inv = 1.0 / (1.0 + 0.5 * dt / tn);
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], wk = B.w[k], e = 0.5 * (uk * uk + vk * vk);
        const double Hop = Ho[r] + fmax(fabs(Ho[r]), kEps * sHo) * (lo[0] + uk * lo[1] + vk * lo[2] + e * lo[3]);
        const double Bop = Bo[r] + 0.5 * fmax(fabs(Bo[r]), kEps * sBo) * lo[3];
        const double Hnp = Hn[r] + fmax(fabs(Hn[r]), kEps * sHn) * (ln[0] + uk * ln[1] + vk * ln[2] + e * ln[3]);
        const double Bnp = Bn[r] + 0.5 * fmax(fabs(Bn[r]), kEps * sBn) * ln[3];
        moment_add(wk, uk, vk, Hop, Bop, acc);
        moment_add(wk, uk, vk, Hnp, Bnp, acc + 4);
        const double hnew = (h[r] + rh[r] + 0.5 * dt * (Hnp / tn + (Hop - h[r]) / to)) * inv;
        const double bnew = (b[r] + rb[r] + 0.5 * dt * (Bnp / tn + (Bop - b[r]) / to)) * inv;
        B.h[(size_t)c * nv + k] = hnew;
        B.b[(size_t)c * nv + k] = bnew;
    }
    block_reduce<8, 0>(acc, red, rout);
    if (tid == 0) {
        const double ro = fmax(fmax(fmax(fabs(to4[0]), fabs(to4[1])), fmax(fabs(to4[2]), fabs(to4[3]))), 1.0);
        const double rn = fmax(fmax(fmax(fabs(Wn[0]), fabs(Wn[1])), fmax(fabs(Wn[2]), fabs(Wn[3]))), 1.0);
        double eo = 0.0, en = 0.0;
        for (int m = 0; m < 4; ++m) { eo = fmax(eo, fabs(acc[m] - to4[m])); en = fmax(en, fabs(acc[4 + m] - Wn[m])); }
        if (!pok || !(eo <= 1.0e-10 * ro) || !(en <= 1.0e-10 * rn)) set_status(B.status, ST_PROJECTION);
        bool fin = true;
        for (int m = 0; m < 4; ++m) { B.W[c * 4 + m] = Wn[m]; fin = fin && isfinite(Wn[m]); }
        if (!fin) set_status(B.status, ST_NONFINITE_STATE);
        // residual-norm contributions (AccumulateMacroResidualNorm, mod_TimeIntegrator.f90:163-191)
        double* dg = B.cell_diag + (size_t)c * kNDiag;
        for (int m = 0; m < 4; ++m) {
            const double d = (Wold[m] - Wn[m]) * P.area / dt;
            dg[m] = d * d;
            dg[4 + m] = fabs(Wn[m]) * P.area;
            dg[9 + m] = fabs(d);
        }
        dg[8] = P.area * P.area;
        bool dok;
        B.dtl[c] = cell_dt(P, Wn, dok);
    }
    last_cta_epilogue(P, B, true, true, red, rout);
}

// -------------------------------------------------------------------------------------------
// InitFlow_Freestream (mod_InitializeFlow.f90:826-856) + the cold-start moment projection
// EnforceAcceptedMomentCompatibility (mod_ImplicitMicro.f90, via InitializeSteadyImplicit).
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX) k_lo_init(LoParams P, LoBuffers B, double rho, double U, double V,
                                                         double tn) {
    __shared__ double red[32 * kRedSlots];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, tid = threadIdx.x, NT = blockDim.x, c = blockIdx.x;
    const Prim p{rho, U, V, 1.0 / tn};
    double W[4];
    get_conserved(P.gm1, p, W);
    const double pref = p.r * (p.L / kPi), bfac = (double)P.ck / (2.0 * p.L);
    double H[VPT], Bm[VPT], acc[14];
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        H[r] = Bm[r] = 0.0;
        if (k >= nv) continue;
        const double dvn = B.u[k] - p.U, dvt = B.v[k] - p.V;
        H[r] = pref * exp(-p.L * (dvn * dvn + dvt * dvt));
        Bm[r] = H[r] * bfac;
        acc[0] = fmax(acc[0], fabs(H[r]));
        acc[1] = fmax(acc[1], fabs(Bm[r]));
    }
    block_reduce<0, 2>(acc, red, rout);
    const double sh = fmax(acc[0], 1.0), sb = fmax(acc[1], 1.0);
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        moment_add(B.w[k], B.u[k], B.v[k], H[r], Bm[r], acc);
        gram_add(B.w[k], fmax(fabs(H[r]), kEps * sh), fmax(fabs(Bm[r]), kEps * sb), B.u[k], B.v[k], acc + 4);
    }
    block_reduce<14, 0>(acc, red, rout);
    double rhs[4], gm[16], lam[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[m] = W[m] - acc[m];
    gram_expand(acc + 4, gm);
    if (!solve_dense4(gm, rhs, lam)) {
        lam[0] = lam[1] = lam[2] = lam[3] = 0.0;
        if (tid == 0) set_status(B.status, ST_PROJECTION);
    }
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const int k = tid + r * NT;
        if (k >= nv) continue;
        const double uk = B.u[k], vk = B.v[k], e = 0.5 * (uk * uk + vk * vk);
        B.h[(size_t)c * nv + k] = H[r] + fmax(fabs(H[r]), kEps * sh) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        B.b[(size_t)c * nv + k] = Bm[r] + 0.5 * fmax(fabs(Bm[r]), kEps * sb) * lam[3];
    }
    if (tid < 4) B.W[c * 4 + tid] = W[tid];
}

// Host-visible launchers (used by ugks_capi.cu).  Tile = (velocities per thread, threads):
// nvel <= 1024 -> (4, <=256 threads); nvel <= 2560 -> (5, <=512 threads).
int lo_vpt(int nvel) { return nvel <= 4 * 256 ? 4 : 5; }

int lo_threads(int nvel) {
    const int vpt = lo_vpt(nvel);
    int t = (nvel + vpt - 1) / vpt;
    t = (t + 31) / 32 * 32;
    return t < 32 ? 32 : t;
}

cudaError_t launch_lo_faces(const LoParams& P, const LoBuffers& B, cudaStream_t s) {
    const int nface = P.nx * P.ny + P.nx * (P.ny - 1) + 2 * P.nx;
    const int nt = lo_threads(P.nvel);
    if (lo_vpt(P.nvel) == 4) k_lo_faces<4, 256><<<nface, nt, 0, s>>>(P, B);
    else k_lo_faces<5, 512><<<nface, nt, 0, s>>>(P, B);
    return cudaGetLastError();
}

template <int VPT, int NTMAX>
static void launch_cells_t(const LoParams& P, const LoBuffers& B, int mode, bool collision, cudaStream_t s) {
    const int nc = P.nx * P.ny, nt = lo_threads(P.nvel);
    if (mode == MODE_FUSED) k_lo_cells<VPT, NTMAX, MODE_FUSED, false><<<nc, nt, 0, s>>>(P, B);
    else if (mode == MODE_UPDATE) k_lo_cells<VPT, NTMAX, MODE_UPDATE, false><<<nc, nt, 0, s>>>(P, B);
    else if (collision) k_lo_cells<VPT, NTMAX, MODE_RESIDUAL, true><<<nc, nt, 0, s>>>(P, B);
    else k_lo_cells<VPT, NTMAX, MODE_RESIDUAL, false><<<nc, nt, 0, s>>>(P, B);
}

cudaError_t launch_lo_cells(const LoParams& P, const LoBuffers& B, int mode, bool collision, cudaStream_t s) {
    if (lo_vpt(P.nvel) == 4) launch_cells_t<4, 256>(P, B, mode, collision, s);
    else launch_cells_t<5, 512>(P, B, mode, collision, s);
    return cudaGetLastError();
}

cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s) {
    k_lo_timestep<<<1, 256, 0, s>>>(P, B);
    return cudaGetLastError();
}

cudaError_t launch_lo_init(const LoParams& P, const LoBuffers& B, double rho, double U, double V, double tn,
                           cudaStream_t s) {
    if (lo_vpt(P.nvel) == 4) k_lo_init<4, 256><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, rho, U, V, tn);
    else k_lo_init<5, 512><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, rho, U, V, tn);
    return cudaGetLastError();
}

}  // namespace ugks
