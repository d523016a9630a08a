// ugks_lo.cu -- second-order UGKS hot path for one Couette domain on sm_100a (FP64).
//
//   k_lo_slopes : Interpolation (mod_Interpolation.f90:26-170): Van-Leer slopes of h and b in x
//                 and y for every (cell, velocity); one-sided slopes on the wall rows.
//   k_lo_faces  : the interior-face flux of EvolutionNative / CalcFlux_MultiDimension
//                 (mod_Evolution.f90:46-177,186-492): one CTA per face.
//   k_lo_walls  : W2BMultiscaleFluxBoundary (mod_Evolution.f90:1888-2449) on the 2*nx wall faces.
//   k_lo_cells  : ComputeResidual (mod_Residual.f90:17-132) + ApplyExplicitUpdate
//                 (mod_TimeIntegrator.f90:16-293) fused, one CTA per cell, plus the next TimeStep
//                 (mod_Solve.f90:373-421) and the residual norms, reduced by the last CTA.
//
// Layout: h, b and the slopes are [cell][velocity] (velocity fastest, coalesced FP64 rows).  A
// CTA covers a whole velocity row, VPT velocities per thread, so every velocity-space moment sum
// is one block reduction.  Velocity loops are branch-free: a thread slot beyond nvel reads a valid
// velocity with weight 0 and skips its stores, so the compiler can interleave the VPT chains.
#include "ugks_lo.cuh"

namespace ugks {

// -------------------------------------------------------------------------------------------
// Interpolation (mod_Interpolation.f90:26-90): slopes sx*, sy* of h and b.  x is periodic; on
// the wall rows the y slope is the one-sided (right-left)/dy of InterpBoundary (:100-117), and
// UnifiedPhysicalOperators skips the Van-Leer inner loop there (:40-45,78-88).
__global__ void __launch_bounds__(256) k_lo_slopes(LoParams P, LoBuffers B) {
    if (eval_cached(B)) return;
    // grid: x covers the velocity row, y = cell; 32-bit index arithmetic only
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    const int c = blockIdx.y, j = c / nx, i = c - j * nx;
    const size_t row = (size_t)nx * nv;
    const size_t idx = (size_t)c * nv + k;
    const size_t cm = (size_t)(j * nx + wrapx(i - 1, nx)) * nv + k, cp = (size_t)(j * nx + wrapx(i + 1, nx)) * nv + k;
    const double h0 = B.h[idx], b0 = B.b[idx];
    B.sxh[idx] = vanleer((h0 - B.h[cm]) * P.inv_dx, (B.h[cp] - h0) * P.inv_dx);
    B.sxb[idx] = vanleer((b0 - B.b[cm]) * P.inv_dx, (B.b[cp] - b0) * P.inv_dx);
    double syh, syb;
    if (j == 0) {
        syh = (B.h[idx + row] - h0) * P.inv_dy;
        syb = (B.b[idx + row] - b0) * P.inv_dy;
    } else if (j == ny - 1) {
        syh = (h0 - B.h[idx - row]) * P.inv_dy;
        syb = (b0 - B.b[idx - row]) * P.inv_dy;
    } else {
        syh = vanleer((h0 - B.h[idx - row]) * P.inv_dy, (B.h[idx + row] - h0) * P.inv_dy);
        syb = vanleer((b0 - B.b[idx - row]) * P.inv_dy, (B.b[idx + row] - b0) * P.inv_dy);
    }
    B.syh[idx] = syh;
    B.syb[idx] = syb;
}

// -------------------------------------------------------------------------------------------
// Interior face: CalcFlux_MultiDimension (mod_Evolution.f90:186-492), UnifiedPhysicalOperators.
// dir 0: vertical face (vn = u, vt = v); dir 1: horizontal face (vn = v, vt = -u).  The upwind
// cell per velocity is the reference's delta = (sign(1,vn)+1)/2 selector (:236-266).
template <int VPT>
__device__ __forceinline__ void lo_face_interior(const LoParams& P, const LoBuffers& B, int dir, int cL, int cR,
                                                 double dt, double* __restrict__ Fh, double* __restrict__ Fb,
                                                 double* Fw, double* red, double* rout, double* sc) {
    const int nv = P.nvel, tid = threadIdx.x;
    const double len = dir == 0 ? P.dx : P.dy;      // cell length normal to the face
    const double flen = dir == 0 ? P.dy : P.dx;     // face length
    const double hl = 0.5 * len;
    const double* sN_h = dir == 0 ? B.sxh : B.syh;
    const double* sN_b = dir == 0 ? B.sxb : B.syb;
    const double* sT_h = dir == 0 ? B.syh : B.sxh;
    const double* sT_b = dir == 0 ? B.syb : B.sxb;
    const double tsg = dir == 0 ? 1.0 : -1.0;       // tangential sign flip on horizontal faces (:262-265)
    double hv[VPT], bv[VPT], H0[VPT];
    double acc[14];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const bool left = copysign(1.0, vn) > 0.0;
        const size_t q = (size_t)(left ? cL : cR) * nv + s.kk;
        const double sg = left ? hl : -hl;
        hv[r] = B.h[q] + sg * sN_h[q];
        bv[r] = B.b[q] + sg * sN_b[q];
        const double sht = tsg * sT_h[q], sbt = tsg * sT_b[q];
        const double v2 = vn * vn + vt * vt;
        acc[0] += wk * hv[r];
        acc[1] += wk * vn * hv[r];
        acc[2] += wk * vt * hv[r];
        acc[3] += 0.5 * wk * (v2 * hv[r] + bv[r]);
        acc[4] += wk * sht;
        acc[5] += wk * vn * sht;
        acc[6] += wk * vt * sht;
        acc[7] += 0.5 * wk * (v2 * sht + sbt);
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    // face state, micro slopes aL, aR, b, A and the time coefficients (GetPrimary, MicroSlope x4,
    // CalcMoment, GetTau, Mt): five independent scalar chains, each run by lane 0 of its own warp so
    // they proceed concurrently, then the time slope A, which needs the first four.  Results go
    // through shared memory: sc[0..3] face prim, [4..19] aL aR b A, [20..24] Mt, [25] Mxi[2],
    // [32..61] the CalcMoment tables, [64..75] the three Moment_auvxi terms of A.
    {
        const int nw = blockDim.x >> 5, w = tid >> 5;
        const bool lane0 = (tid & 31) == 0;
        Prim pf;
        const double cv[4] = {rout[0], rout[1], rout[2], rout[3]};
        const bool ok = get_primary(P.gm1, cv, pf);
        if (!ok) { pf.r = 1.0; pf.U = 0.0; pf.V = 0.0; pf.L = 1.0; }
        if (lane0) {
            for (int piece = w; piece < 5; piece += nw) {
                if (piece <= 1) {            // aL from (W_face - W_L) / (dx/2), aR from (W_R - W_face) / (dx/2)
                    const double* Wc = B.W + (piece == 0 ? cL : cR) * 4;
                    double wc[4], sw[4], a4[4];
                    wc[0] = Wc[0]; wc[3] = Wc[3];
                    if (dir == 0) { wc[1] = Wc[1]; wc[2] = Wc[2]; }
                    else { wc[1] = Wc[2]; wc[2] = -Wc[1]; }
#pragma unroll
                    for (int m = 0; m < 4; ++m) sw[m] = piece == 0 ? (cv[m] - wc[m]) / hl : (wc[m] - cv[m]) / hl;
                    micro_slope(P.ck, pf, sw, a4);
#pragma unroll
                    for (int m = 0; m < 4; ++m) sc[4 + 4 * piece + m] = a4[m];
                    if (piece == 0) {
                        sc[0] = pf.r; sc[1] = pf.U; sc[2] = pf.V; sc[3] = pf.L;
                        if (!ok) set_status(B.status, ST_GETPRIMARY);
                    }
                } else if (piece == 2) {     // b from the tangential slope moments
                    const double swt[4] = {rout[4], rout[5], rout[6], rout[7]};
                    double a4[4];
                    micro_slope(P.ck, pf, swt, a4);
#pragma unroll
                    for (int m = 0; m < 4; ++m) sc[12 + m] = a4[m];
                } else if (piece == 3) {     // CalcMoment tables
                    Moments M;
                    calc_moment(P.ck, pf, M);
#pragma unroll
                    for (int m = 0; m <= kMNUM; ++m) { sc[32 + m] = M.Mu[m]; sc[39 + m] = M.MuL[m]; sc[46 + m] = M.MuR[m]; }
#pragma unroll
                    for (int m = 0; m <= kMTUM; ++m) sc[53 + m] = M.Mv[m];
#pragma unroll
                    for (int m = 0; m < 3; ++m) sc[59 + m] = M.Mxi[m];
                    sc[25] = M.Mxi[2];
                } else {                     // GetTau and Mt(1..5)
                    double tau = 1.0, Mt[5];
                    const bool tok = get_tau(P.mu_ref, P.omega, pf, tau);
                    if (!tok) tau = 1.0;
                    time_coeffs(dt, tau, Mt);
#pragma unroll
                    for (int m = 0; m < 5; ++m) sc[20 + m] = Mt[m];
                    if (ok && !tok) set_status(B.status, ST_TAU);
                }
            }
        }
        __syncthreads();
        if (lane0) {
            for (int piece = w; piece < 3; piece += nw) {   // Moment_auvxi of aL (MuL), aR (MuR), b (Mu, v)
                double a4[4], o4[4];
#pragma unroll
                for (int m = 0; m < 4; ++m) a4[m] = sc[4 + 4 * piece + m];
                const double* Mu = sc + (piece == 0 ? 39 : (piece == 1 ? 46 : 32));
                moment_auvxi(a4, Mu, sc + 53, sc + 59, piece == 2 ? 0 : 1, piece == 2 ? 1 : 0, o4);
#pragma unroll
                for (int m = 0; m < 4; ++m) sc[64 + 4 * piece + m] = o4[m];
            }
        }
        __syncthreads();
        if (tid == 0) {
            double sw[4], aT[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) sw[m] = -pf.r * (sc[64 + m] + sc[68 + m] + sc[72 + m]);
            micro_slope(P.ck, pf, sw, aT);
#pragma unroll
            for (int m = 0; m < 4; ++m) sc[16 + m] = aT[m];
        }
    }
    __syncthreads();
    const Prim pf{sc[0], sc[1], sc[2], sc[3]};
    double aL[4], aR[4], bs[4], aT[4], Mt[5];
#pragma unroll
    for (int m = 0; m < 4; ++m) { aL[m] = sc[4 + m]; aR[m] = sc[8 + m]; bs[m] = sc[12 + m]; aT[m] = sc[16 + m]; }
#pragma unroll
    for (int m = 0; m < 5; ++m) Mt[m] = sc[20 + m];
    const double mxi2 = sc[25];
    // face equilibrium H0 (PrepareNativeFaceEquilibrium, mod_Evolution.f90:16-30) + heat flux
    const double pref = pf.r * (pf.L / kPi), bfac = (double)P.ck / (2.0 * pf.L);
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const double dvn = vn - pf.U, dvt = vt - pf.V, v2 = dvn * dvn + dvt * dvt;
        H0[r] = pref * exp(-pf.L * v2);
        const double t = 0.5 * wk * (v2 * hv[r] + bv[r]);
        acc[0] += t * dvn;
        acc[1] += t * dvt;
        acc[2] = fmax(acc[2], s.ok ? fabs(H0[r]) : 0.0);
        acc[3] = fmax(acc[3], s.ok ? fabs(H0[r] * bfac) : 0.0);
    }
    block_reduce<2, 2>(acc, red, rout);
    const double qf0 = acc[0], qf1 = acc[1];
    const double sch = fmax(acc[2], 1.0), scb = fmax(acc[3], 1.0);
    // ProjectToConservedMoments of (H0, B0) onto GetConserved(pf), local frame (mod_ImplicitCommon.f90:42-82)
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const double b0 = H0[r] * bfac;
        moment_add(wk, vn, vt, H0[r], b0, acc);
        gram_add(wk, fmax(fabs(H0[r]), kEps * sch), fmax(fabs(b0), kEps * scb), vn, vt, acc + 4);
    }
    block_reduce_smem<14, 0>(acc, red, rout);
    double tgt[4], lam[4];
    get_conserved(P.gm1, pf, tgt);
    if (tid == 0) {   // SolveDense4 once per face, broadcast
        double rhs[4], gm[16], l[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = tgt[m] - rout[m];
        gram_expand(rout + 4, gm);
        if (!solve_dense4(gm, rhs, l)) {
            l[0] = l[1] = l[2] = l[3] = 0.0;
            set_status(B.status, ST_FACE_PROJECTION);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[26 + m] = l[m];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 4; ++m) lam[m] = sc[26 + m];
    // Shakhov part and the micro flux (mod_Evolution.f90:396-453), times the face length.
    const double coeff = 0.8 * (1.0 - P.pr) * pf.L * pf.L / pf.r;
    const double c2ck = 2.0 / (double)P.ck;
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double a = dir == 0 ? uk : vk, t = dir == 0 ? vk : -uk;
        const double b0 = H0[r] * bfac;
        const double e = 0.5 * (a * a + t * t);
        const double H = H0[r] + fmax(fabs(H0[r]), kEps * sch) * (lam[0] + a * lam[1] + t * lam[2] + e * lam[3]);
        const double Bq = b0 + 0.5 * fmax(fabs(b0), kEps * scb) * lam[3];
        moment_add(wk, a, t, H, Bq, acc);   // projection gate
        const bool left = copysign(1.0, a) > 0.0;
        const size_t q = (size_t)(left ? cL : cR) * nv + s.kk;
        const double shn = sN_h[q], sbn = sN_b[q], sht = tsg * sT_h[q], sbt = tsg * sT_b[q];
        const double dvn = a - pf.U, dvt = t - pf.V, dv2 = dvn * dvn + dvt * dvt;
        const double qdot = dvn * qf0 + dvt * qf1;
        const double shH = 2.0 * pf.L * dv2 - 4.0;
        const double Hp = coeff * qdot * shH * H, Bp = coeff * qdot * (shH + c2ck) * Bq;
        const double v2 = a * a + t * t;
        const double slh = a * shn + t * sht, slb = a * sbn + t * sbt;
        const double* as = left ? aL : aR;
        const double h_a = as[0] * H + as[1] * a * H + as[2] * t * H + 0.5 * as[3] * (v2 * H + Bq);
        const double h_b = bs[0] * H + bs[1] * a * H + bs[2] * t * H + 0.5 * bs[3] * (v2 * H + Bq);
        const double h_T = aT[0] * H + aT[1] * a * H + aT[2] * t * H + 0.5 * aT[3] * (v2 * H + Bq);
        const double b_a = as[0] * Bq + as[1] * a * Bq + as[2] * t * Bq + 0.5 * as[3] * (v2 * Bq + mxi2 * H);
        const double b_b = bs[0] * Bq + bs[1] * a * Bq + bs[2] * t * Bq + 0.5 * bs[3] * (v2 * Bq + mxi2 * H);
        const double b_T = aT[0] * Bq + aT[1] * a * Bq + aT[2] * t * Bq + 0.5 * aT[3] * (v2 * Bq + mxi2 * H);
        const double fh = Mt[0] * a * (H + Hp) + Mt[1] * a * a * h_a + Mt[1] * a * t * h_b + Mt[2] * a * h_T +
                          Mt[3] * a * hv[r] - Mt[4] * a * slh;
        const double fb = Mt[0] * a * (Bq + Bp) + Mt[1] * a * a * b_a + Mt[1] * a * t * b_b + Mt[2] * a * b_T +
                          Mt[3] * a * bv[r] - Mt[4] * a * slb;
        const double Fhk = flen * fh, Fbk = flen * fb;
        if (s.ok) { Fh[s.k] = Fhk; Fb[s.k] = Fbk; }
        moment_add(wk, uk, vk, Fhk, Fbk, acc + 4);   // MomentConserved in the global frame (:470-473)
    }
    block_reduce<8, 0>(acc, red, rout);
    if (tid == 0) {
        const double rs = fmax(fmax(fmax(fabs(tgt[0]), fabs(tgt[1])), fmax(fabs(tgt[2]), fabs(tgt[3]))), 1.0);
        double err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) err = fmax(err, fabs(acc[m] - tgt[m]));
        if (!(err <= 1.0e-10 * rs)) set_status(B.status, ST_FACE_PROJECTION);
        bool fin = true;
#pragma unroll
        for (int m = 0; m < 4; ++m) { Fw[m] = acc[4 + m]; fin = fin && isfinite(acc[4 + m]); }
        if (!fin) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// -------------------------------------------------------------------------------------------
// Interior face on WPF warps (nvel <= 1024): the arithmetic of lo_face_interior, with every velocity
// sum a per-lane sum over the thread's velocities k = t, t + 32 WPF, ... (t = the thread's index in the
// face) followed by a warp butterfly and, for WPF > 1, the sum of the WPF warp totals in warp order,
// which every thread of the face holds.  The face's scalar chain (GetPrimary, MicroSlope x4, CalcMoment,
// GetTau, Mt) then runs on every thread alike, so no thread waits on another's serial phase; H0 of the
// thread's velocities waits in shared memory (sH[k]) between the passes that use it.

// totals of v over the face: every thread of the face holds them.  WPF = 1: the warp butterfly; WPF > 1:
// one face per CTA, the warps' totals exchanged through xch [WPF][32]
template <int N, int WPF, bool MAX = false>
__device__ __forceinline__ void face_reduce_all(double* v, double* xch) {
    if constexpr (WPF == 1) {
        if constexpr (MAX) warp_max_all<N>(v);
        else warp_sum_all<N>(v);
    } else {
        constexpr int sh = 5 - ilog2(pow2_ceil(N));
        const double r = warp_halving<N, MAX>(v);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if ((lane & ((1 << sh) - 1)) == 0 && (lane >> sh) < N) xch[w * 32 + (lane >> sh)] = r;
        __syncthreads();
#pragma unroll
        for (int q = 0; q < N; ++q) {
            double t = xch[q];
#pragma unroll
            for (int ww = 1; ww < WPF; ++ww) t = MAX ? fmax(t, xch[ww * 32 + q]) : t + xch[ww * 32 + q];
            v[q] = t;
        }
        __syncthreads();   // xch is rewritten by the next reduction
    }
}

template <int WPF>
__device__ __forceinline__ void lo_face_interior_grp(const LoParams& P, const LoBuffers& B, int dir, int cL, int cR,
                                                     double dt, double* __restrict__ Fh, double* __restrict__ Fb,
                                                     double* Fw, double* sH, double* xch) {
    constexpr int NT = 32 * WPF;
    const int nv = P.nvel, lane = WPF == 1 ? (threadIdx.x & 31) : (int)threadIdx.x, nr = (nv + NT - 1) / NT;
    const bool lead = lane == 0;
    const double len = dir == 0 ? P.dx : P.dy, flen = dir == 0 ? P.dy : P.dx, hl = 0.5 * len;
    const double* sN_h = dir == 0 ? B.sxh : B.syh;
    const double* sN_b = dir == 0 ? B.sxb : B.syb;
    const double* sT_h = dir == 0 ? B.syh : B.sxh;
    const double* sT_b = dir == 0 ? B.syb : B.sxb;
    const double tsg = dir == 0 ? 1.0 : -1.0;
    double acc[14];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll 4
    for (int r = 0; r < nr; ++r) {
        const int k = lane + NT * r;
        const bool kok = k < nv;
        const int kk = kok ? k : nv - 1;
        const double uk = B.u[kk], vk = B.v[kk], wk = kok ? B.w[kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const bool left = copysign(1.0, vn) > 0.0;
        const size_t q = (size_t)(left ? cL : cR) * nv + kk;
        const double sg = left ? hl : -hl;
        const double hv = B.h[q] + sg * sN_h[q], bv = B.b[q] + sg * sN_b[q];
        const double sht = tsg * sT_h[q], sbt = tsg * sT_b[q];
        const double v2 = vn * vn + vt * vt;
        acc[0] += wk * hv;
        acc[1] += wk * vn * hv;
        acc[2] += wk * vt * hv;
        acc[3] += 0.5 * wk * (v2 * hv + bv);
        acc[4] += wk * sht;
        acc[5] += wk * vn * sht;
        acc[6] += wk * vt * sht;
        acc[7] += 0.5 * wk * (v2 * sht + sbt);
    }
    face_reduce_all<8, WPF>(acc, xch);
    // the face's scalar chain, on every thread
    Prim pf;
    const double cv[4] = {acc[0], acc[1], acc[2], acc[3]};
    const bool ok = get_primary(P.gm1, cv, pf);
    if (!ok) { pf.r = 1.0; pf.U = 0.0; pf.V = 0.0; pf.L = 1.0; }
    double aL[4], aR[4], bs[4], aT[4], Mt[5];
    for (int piece = 0; piece < 2; ++piece) {   // aL from (W_face - W_L) / (dx/2), aR from (W_R - W_face) / (dx/2)
        const double* Wc = B.W + (piece == 0 ? cL : cR) * 4;
        double wc[4], sw[4];
        wc[0] = Wc[0]; wc[3] = Wc[3];
        if (dir == 0) { wc[1] = Wc[1]; wc[2] = Wc[2]; }
        else { wc[1] = Wc[2]; wc[2] = -Wc[1]; }
#pragma unroll
        for (int m = 0; m < 4; ++m) sw[m] = piece == 0 ? (cv[m] - wc[m]) / hl : (wc[m] - cv[m]) / hl;
        micro_slope(P.ck, pf, sw, piece == 0 ? aL : aR);
    }
    {
        const double swt[4] = {acc[4], acc[5], acc[6], acc[7]};
        micro_slope(P.ck, pf, swt, bs);
    }
    Moments M;
    calc_moment(P.ck, pf, M);
    double tau = 1.0;
    const bool tok = get_tau(P.mu_ref, P.omega, pf, tau);
    if (!tok) tau = 1.0;
    time_coeffs(dt, tau, Mt);
    if (lead) {
        if (!ok) set_status(B.status, ST_GETPRIMARY);
        if (ok && !tok) set_status(B.status, ST_TAU);
    }
    {
        double o0[4], o1[4], o2[4], sw[4];
        moment_auvxi(aL, M.MuL, M.Mv, M.Mxi, 1, 0, o0);
        moment_auvxi(aR, M.MuR, M.Mv, M.Mxi, 1, 0, o1);
        moment_auvxi(bs, M.Mu, M.Mv, M.Mxi, 0, 1, o2);
#pragma unroll
        for (int m = 0; m < 4; ++m) sw[m] = -pf.r * (o0[m] + o1[m] + o2[m]);
        micro_slope(P.ck, pf, sw, aT);
    }
    const double mxi2 = M.Mxi[2];
    // face equilibrium H0 (PrepareNativeFaceEquilibrium, mod_Evolution.f90:16-30) + heat flux
    const double pref = pf.r * (pf.L / kPi), bfac = (double)P.ck / (2.0 * pf.L);
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll 4
    for (int r = 0; r < nr; ++r) {
        const int k = lane + NT * r;
        const bool kok = k < nv;
        const int kk = kok ? k : nv - 1;
        const double uk = B.u[kk], vk = B.v[kk], wk = kok ? B.w[kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const bool left = copysign(1.0, vn) > 0.0;
        const size_t q = (size_t)(left ? cL : cR) * nv + kk;
        const double sg = left ? hl : -hl;
        const double hv = B.h[q] + sg * sN_h[q], bv = B.b[q] + sg * sN_b[q];
        const double dvn = vn - pf.U, dvt = vt - pf.V, v2 = dvn * dvn + dvt * dvt;
        const double H0 = pref * exp(-pf.L * v2);
        sH[k] = H0;
        const double t = 0.5 * wk * (v2 * hv + bv);
        acc[0] += t * dvn;
        acc[1] += t * dvt;
        acc[2] = fmax(acc[2], kok ? fabs(H0) : 0.0);
        acc[3] = fmax(acc[3], kok ? fabs(H0 * bfac) : 0.0);
    }
    face_reduce_all<2, WPF>(acc, xch);
    face_reduce_all<2, WPF, true>(acc + 2, xch);
    const double qf0 = acc[0], qf1 = acc[1];
    const double sch = fmax(acc[2], 1.0), scb = fmax(acc[3], 1.0);
    // ProjectToConservedMoments of (H0, B0) onto GetConserved(pf), local frame (mod_ImplicitCommon.f90:42-82)
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll 4
    for (int r = 0; r < nr; ++r) {
        const int k = lane + NT * r;
        const bool kok = k < nv;
        const int kk = kok ? k : nv - 1;
        const double uk = B.u[kk], vk = B.v[kk], wk = kok ? B.w[kk] : 0.0;
        const double vn = dir == 0 ? uk : vk, vt = dir == 0 ? vk : -uk;
        const double H0 = sH[k], b0 = H0 * bfac;
        moment_add(wk, vn, vt, H0, b0, acc);
        gram_add(wk, fmax(fabs(H0), kEps * sch), fmax(fabs(b0), kEps * scb), vn, vt, acc + 4);
    }
    face_reduce_all<14, WPF>(acc, xch);
    double tgt[4], lam[4];
    get_conserved(P.gm1, pf, tgt);
    {
        double rhs[4], gm[16];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = tgt[m] - acc[m];
        gram_expand(acc + 4, gm);
        if (!solve_dense4(gm, rhs, lam)) {
            lam[0] = lam[1] = lam[2] = lam[3] = 0.0;
            if (lead) set_status(B.status, ST_FACE_PROJECTION);
        }
    }
    // Shakhov part and the micro flux (mod_Evolution.f90:396-453), times the face length
    const double coeff = 0.8 * (1.0 - P.pr) * pf.L * pf.L / pf.r;
    const double c2ck = 2.0 / (double)P.ck;
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll 2
    for (int r = 0; r < nr; ++r) {
        const int k = lane + NT * r;
        const bool kok = k < nv;
        const int kk = kok ? k : nv - 1;
        const double uk = B.u[kk], vk = B.v[kk], wk = kok ? B.w[kk] : 0.0;
        const double a = dir == 0 ? uk : vk, t = dir == 0 ? vk : -uk;
        const double H0 = sH[k], b0 = H0 * bfac;
        const double e = 0.5 * (a * a + t * t);
        const double H = H0 + fmax(fabs(H0), kEps * sch) * (lam[0] + a * lam[1] + t * lam[2] + e * lam[3]);
        const double Bq = b0 + 0.5 * fmax(fabs(b0), kEps * scb) * lam[3];
        moment_add(wk, a, t, H, Bq, acc);   // projection gate
        const bool left = copysign(1.0, a) > 0.0;
        const size_t q = (size_t)(left ? cL : cR) * nv + kk;
        const double sg = left ? hl : -hl;
        const double shn = sN_h[q], sbn = sN_b[q], sht = tsg * sT_h[q], sbt = tsg * sT_b[q];
        const double hv = B.h[q] + sg * shn, bv = B.b[q] + sg * sbn;
        const double dvn = a - pf.U, dvt = t - pf.V, dv2 = dvn * dvn + dvt * dvt;
        const double qdot = dvn * qf0 + dvt * qf1;
        const double shH = 2.0 * pf.L * dv2 - 4.0;
        const double Hp = coeff * qdot * shH * H, Bp = coeff * qdot * (shH + c2ck) * Bq;
        const double v2 = a * a + t * t;
        const double slh = a * shn + t * sht, slb = a * sbn + t * sbt;
        const double* as = left ? aL : aR;
        const double h_a = as[0] * H + as[1] * a * H + as[2] * t * H + 0.5 * as[3] * (v2 * H + Bq);
        const double h_b = bs[0] * H + bs[1] * a * H + bs[2] * t * H + 0.5 * bs[3] * (v2 * H + Bq);
        const double h_T = aT[0] * H + aT[1] * a * H + aT[2] * t * H + 0.5 * aT[3] * (v2 * H + Bq);
        const double b_a = as[0] * Bq + as[1] * a * Bq + as[2] * t * Bq + 0.5 * as[3] * (v2 * Bq + mxi2 * H);
        const double b_b = bs[0] * Bq + bs[1] * a * Bq + bs[2] * t * Bq + 0.5 * bs[3] * (v2 * Bq + mxi2 * H);
        const double b_T = aT[0] * Bq + aT[1] * a * Bq + aT[2] * t * Bq + 0.5 * aT[3] * (v2 * Bq + mxi2 * H);
        const double fh = Mt[0] * a * (H + Hp) + Mt[1] * a * a * h_a + Mt[1] * a * t * h_b + Mt[2] * a * h_T +
                          Mt[3] * a * hv - Mt[4] * a * slh;
        const double fb = Mt[0] * a * (Bq + Bp) + Mt[1] * a * a * b_a + Mt[1] * a * t * b_b + Mt[2] * a * b_T +
                          Mt[3] * a * bv - Mt[4] * a * slb;
        const double Fhk = flen * fh, Fbk = flen * fb;
        if (kok) { Fh[k] = Fhk; Fb[k] = Fbk; }
        moment_add(wk, uk, vk, Fhk, Fbk, acc + 4);   // MomentConserved in the global frame (:470-473)
    }
    face_reduce_all<8, WPF>(acc, xch);
    if (lead) {
        const double rs = fmax(fmax(fmax(fabs(tgt[0]), fabs(tgt[1])), fmax(fabs(tgt[2]), fabs(tgt[3]))), 1.0);
        double err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) err = fmax(err, fabs(acc[m] - tgt[m]));
        if (!(err <= 1.0e-10 * rs)) set_status(B.status, ST_FACE_PROJECTION);
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
__device__ __forceinline__ void lo_face_wall(const LoParams& P, const LoBuffers& B, int side, int i, double dt,
                                             double* __restrict__ Fh, double* __restrict__ Fb, double* Fw,
                                             double* aero, double* red, double* rout) {
    const int nv = P.nvel, tid = threadIdx.x;
    const int iw = side < 0 ? 0 : 1;
    const int j = side < 0 ? 0 : P.ny - 1;
    const int cell = j * P.nx + i;
    const double len = P.dy, flen = P.dx;
    const double rot = -(double)side;
    double hv[VPT], bv[VPT], Hg[VPT], Hw[VPT];
    const double* Wc = B.W + cell * 4;
    Prim pc;
    const bool ok = get_primary(P.gm1, Wc, pc);
    // LocalFrame with cosx = -0, cosy = 1 (mod_Tools.f90:150-162): (r, U, V) -> (r, V, -U)
    const Prim prim{pc.r, pc.V, -pc.U, pc.L};
    const Prim pw{1.0, P.wall_ux[iw] * (-0.0) + 0.0 * 1.0, -P.wall_ux[iw] * 1.0 + 0.0 * (-0.0), P.wall_lam[iw]};
    Prim pg = pw;
    pg.r = prim.r / prim.L * pw.L;   // keep the cell pressure (:2027)
    double tau = 1.0, Mt[5];
    const bool tok = get_tau(P.mu_ref, P.omega, pg, tau);
    if (!tok) tau = 1.0;
    time_coeffs(dt, tau, Mt);
    if (tid == 0) {
        if (!ok) set_status(B.status, ST_GETPRIMARY);
        if (ok && !tok) set_status(B.status, ST_TAU);
    }
    const double prefg = pg.r * (pg.L / kPi), prefw = 1.0 * (pw.L / kPi), bfac = (double)P.ck / (2.0 * pw.L);
    double acc[28];
#pragma unroll
    for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double vn = vk, vt = -uk;
        const size_t q = (size_t)cell * nv + s.kk;
        const double sht = -B.sxh[q], sbt = -B.sxb[q];
        hv[r] = B.h[q] - rot * 0.5 * len * B.syh[q];
        bv[r] = B.b[q] - rot * 0.5 * len * B.syb[q];
        const double dvn = vn - pg.U, dvt = vt - pg.V, v2 = dvn * dvn + dvt * dvt;
        const double ex = exp(-pg.L * v2);
        Hg[r] = prefg * ex;
        Hw[r] = prefw * ex;
        const double lv2 = vn * vn + vt * vt;
        acc[0] += wk * sht;
        acc[1] += wk * vn * sht;
        acc[2] += wk * vt * sht;
        acc[3] += 0.5 * wk * (lv2 * sht + sbt);
        acc[4] += 0.5 * wk * dvn * (v2 * hv[r] + bv[r]);
        acc[5] += 0.5 * wk * dvt * (v2 * hv[r] + bv[r]);
        acc[6] = fmax(acc[6], s.ok ? fabs(Hg[r]) : 0.0);
        acc[7] = fmax(acc[7], s.ok ? fabs(Hg[r] * bfac) : 0.0);
        acc[8] = fmax(acc[8], s.ok ? fabs(Hw[r]) : 0.0);
        acc[9] = fmax(acc[9], s.ok ? fabs(Hw[r] * bfac) : 0.0);
    }
    block_reduce<6, 4>(acc, red, rout);
    const double swt[4] = {acc[0], acc[1], acc[2], acc[3]};
    const double qf0 = acc[4], qf1 = acc[5];
    const double sgh = fmax(acc[6], 1.0), sgb = fmax(acc[7], 1.0), swh = fmax(acc[8], 1.0), swb = fmax(acc[9], 1.0);
    // micro slopes a_gn, a_gt, a_T (mod_Evolution.f90:2044-2087)
    double cg[4], a_gn[4], a_gt[4], a_T[4], sw[4], mxi2;
    get_conserved(P.gm1, pg, cg);
    const double cg1[4] = {Wc[0], Wc[2], -Wc[1], Wc[3]};
#pragma unroll
    for (int m = 0; m < 4; ++m) sw[m] = (cg[m] - cg1[m]) / ((double)side * 0.5 * len);
    micro_slope(P.ck, pg, sw, a_gn);
    micro_slope(P.ck, pg, swt, a_gt);
    {
        Moments M;
        calc_moment(P.ck, pg, M);
        double Mau[4], Mbv[4];
        moment_auvxi(a_gn, M.Mu, M.Mv, M.Mxi, 1, 0, Mau);
        moment_auvxi(a_gt, M.Mu, M.Mv, M.Mxi, 0, 1, Mbv);
#pragma unroll
        for (int m = 0; m < 4; ++m) sw[m] = -pg.r * (Mau[m] + Mbv[m]);
        micro_slope(P.ck, pg, sw, a_T);
        mxi2 = M.Mxi[2];
    }
    // the two face-equilibrium projections: H_g onto GetConserved(pg), H_w onto GetConserved(pshape)
#pragma unroll
    for (int m = 0; m < 28; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double vn = vk, vt = -uk;
        const double bg = Hg[r] * bfac, bw = Hw[r] * bfac;
        moment_add(wk, vn, vt, Hg[r], bg, acc);
        gram_add(wk, fmax(fabs(Hg[r]), kEps * sgh), fmax(fabs(bg), kEps * sgb), vn, vt, acc + 4);
        moment_add(wk, vn, vt, Hw[r], bw, acc + 14);
        gram_add(wk, fmax(fabs(Hw[r]), kEps * swh), fmax(fabs(bw), kEps * swb), vn, vt, acc + 18);
    }
    block_reduce<28, 0>(acc, red, rout);
    double tg[4], tw[4], lg[4], lw[4];
    const Prim pshape{1.0, pw.U, pw.V, pw.L};
    get_conserved(P.gm1, pg, tg);
    get_conserved(P.gm1, pshape, tw);
    bool pok;
    {
        double rhs[4], gm[16];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = tg[m] - acc[m];
        gram_expand(acc + 4, gm);
        pok = solve_dense4(gm, rhs, lg);
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = tw[m] - acc[14 + m];
        gram_expand(acc + 18, gm);
        pok = solve_dense4(gm, rhs, lw) && pok;
    }
    if (!pok) { lg[0] = lg[1] = lg[2] = lg[3] = lw[0] = lw[1] = lw[2] = lw[3] = 0.0; }
    const double coeff = 0.8 * (1.0 - P.pr) * pg.L * pg.L / pg.r;
    const double c2ck = 2.0 / (double)P.ck;
    double Bg[VPT], Bw[VPT];
#pragma unroll
    for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double a = vk, t = -uk, e = 0.5 * (a * a + t * t);
        const double bg = Hg[r] * bfac, bw = Hw[r] * bfac;
        Hg[r] = Hg[r] + fmax(fabs(Hg[r]), kEps * sgh) * (lg[0] + a * lg[1] + t * lg[2] + e * lg[3]);
        Bg[r] = bg + 0.5 * fmax(fabs(bg), kEps * sgb) * lg[3];
        Hw[r] = Hw[r] + fmax(fabs(Hw[r]), kEps * swh) * (lw[0] + a * lw[1] + t * lw[2] + e * lw[3]);
        Bw[r] = bw + 0.5 * fmax(fabs(bw), kEps * swb) * lw[3];
        moment_add(wk, a, t, Hg[r], Bg[r], acc + 2);
        moment_add(wk, a, t, Hw[r], Bw[r], acc + 6);
        const double dk = (copysign(1.0, a) * rot + 1.0) / 2.0, ik = 1.0 - dk;
        const size_t q = (size_t)cell * nv + s.kk;
        const double slh = a * B.syh[q] + t * (-B.sxh[q]);
        const double v2 = a * a + t * t;
        const double dvn = a - pg.U, dvt = t - pg.V, dv2 = dvn * dvn + dvt * dvt;
        const double Hp = coeff * (dvn * qf0 + dvt * qf1) * (2.0 * pg.L * dv2 - 4.0) * Hg[r];
        const double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hg[r] + 0.5 * a_gn[3] * (v2 * Hg[r] + Bg[r]);
        const double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hg[r] + 0.5 * a_gt[3] * (v2 * Hg[r] + Bg[r]);
        const double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hg[r] + 0.5 * a_T[3] * (v2 * Hg[r] + Bg[r]);
        acc[0] += wk * a * ik * (Mt[0] * (Hg[r] + Hp) + Mt[1] * (a * Ha_gn + t * Ha_gt) + Mt[2] * Ha_T +
                                 Mt[3] * hv[r] - Mt[4] * slh);
        acc[1] += wk * a * Hw[r] * dk;
    }
    block_reduce<10, 0>(acc, red, rout);
    const double rhow = -acc[0] / (dt * acc[1]);   // prim_w(1) = -incidence/reflection (:2166)
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
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double a = vk, t = -uk, v2 = a * a + t * t;
        const double dk = (copysign(1.0, a) * rot + 1.0) / 2.0, ik = 1.0 - dk;
        const size_t q = (size_t)cell * nv + s.kk;
        const double shn = B.syh[q], sbn = B.syb[q], sht = -B.sxh[q], sbt = -B.sxb[q];
        const double Hwk = rhow * Hw[r], Bwk = rhow * Bw[r];
        const double Hgk = Hg[r], Bgk = Bg[r];
        const double dvn = a - pg.U, dvt = t - pg.V, dv2 = dvn * dvn + dvt * dvt;
        const double qdot = dvn * qf0 + dvt * qf1;
        const double shH = 2.0 * pg.L * dv2 - 4.0;
        const double Hp = coeff * qdot * shH * Hgk, Bp = coeff * qdot * (shH + c2ck) * Bgk;
        const double Ha_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Hgk + 0.5 * a_gn[3] * (v2 * Hgk + Bgk);
        const double Ha_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Hgk + 0.5 * a_gt[3] * (v2 * Hgk + Bgk);
        const double Ha_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Hgk + 0.5 * a_T[3] * (v2 * Hgk + Bgk);
        const double Ba_gn = (a_gn[0] + a_gn[1] * a + a_gn[2] * t) * Bgk + 0.5 * a_gn[3] * (v2 * Bgk + mxi2 * Hgk);
        const double Ba_gt = (a_gt[0] + a_gt[1] * a + a_gt[2] * t) * Bgk + 0.5 * a_gt[3] * (v2 * Bgk + mxi2 * Hgk);
        const double Ba_T = (a_T[0] + a_T[1] * a + a_T[2] * t) * Bgk + 0.5 * a_T[3] * (v2 * Bgk + mxi2 * Hgk);
        const double fh = flen * (dt * a * Hwk * dk + Mt[0] * a * (Hgk + Hp) * ik + Mt[1] * a * a * Ha_gn * ik +
                                  Mt[1] * a * t * Ha_gt * ik + Mt[2] * a * Ha_T * ik + Mt[3] * a * hv[r] * ik -
                                  Mt[4] * a * (a * shn + t * sht) * ik);
        const double fb = flen * (dt * a * Bwk * dk + Mt[0] * a * (Bgk + Bp) * ik + Mt[1] * a * a * Ba_gn * ik +
                                  Mt[1] * a * t * Ba_gt * ik + Mt[2] * a * Ba_T * ik + Mt[3] * a * bv[r] * ik -
                                  Mt[4] * a * (a * sbn + t * sbt) * ik);
        if (s.ok) { Fh[s.k] = fh; Fb[s.k] = fb; }
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
        // GlobalFrame with cosx = -0, cosy = 1: (f1, f2, f3, f4) -> (f1, -f3, f2, f4), times the face length
        Fw[0] = flen * acc[0];
        Fw[1] = flen * (-acc[2]);
        Fw[2] = flen * acc[1];
        Fw[3] = flen * acc[3];
        if (!(isfinite(acc[0]) && isfinite(acc[1]) && isfinite(acc[2]) && isfinite(acc[3])))
            set_status(B.status, ST_NONFINITE_FLUX);
    }
}

template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_lo_faces(LoParams P, LoBuffers B) {
    if (eval_cached(B)) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[80];
    const double dt = B.dt[0];
    const int nx = P.nx, ny = P.ny, nv = P.nvel;
    int f = blockIdx.x;
    if (f < nx * ny) {
        const int j = f / nx, i = f % nx;
        const size_t o = (size_t)(j * nx + i);
        lo_face_interior<VPT>(P, B, 0, j * nx + wrapx(i - 1, nx), j * nx + i, dt, B.fxh + o * nv, B.fxb + o * nv,
                              B.fxw + o * 4, red, rout, sc);
        return;
    }
    f -= nx * ny;
    const int jf = 1 + f / nx, i = f % nx;
    const size_t o = (size_t)(jf * nx + i);
    lo_face_interior<VPT>(P, B, 1, (jf - 1) * nx + i, jf * nx + i, dt, B.fyh + o * nv, B.fyb + o * nv, B.fyw + o * 4,
                          red, rout, sc);
}

// the interior faces (x faces, then the y faces between rows) on WPF warps each: NF faces per CTA when
// WPF = 1, one when WPF > 1; nvel <= 1024
template <int NF, int WPF>
__global__ void __launch_bounds__(NF * WPF * 32) k_lo_faces_grp(LoParams P, LoBuffers B) {
    static_assert(NF == 1 || WPF == 1, "several faces per CTA only with one warp each");
    if (eval_cached(B)) return;
    __shared__ double sH[NF][1024];
    __shared__ double xch[WPF > 1 ? WPF * 32 : 1];
    const double dt = B.dt[0];
    const int nx = P.nx, ny = P.ny, nv = P.nvel, w = NF == 1 ? 0 : (int)(threadIdx.x >> 5);
    int f = blockIdx.x * NF + w;
    if (f >= nx * ny + nx * (ny - 1)) return;   // only when NF > 1 (no face-wide barrier then)
    if (f < nx * ny) {
        const int j = f / nx, i = f % nx;
        const size_t o = (size_t)(j * nx + i);
        lo_face_interior_grp<WPF>(P, B, 0, j * nx + wrapx(i - 1, nx), j * nx + i, dt, B.fxh + o * nv, B.fxb + o * nv,
                                  B.fxw + o * 4, sH[w], xch);
        return;
    }
    f -= nx * ny;
    const int jf = 1 + f / nx, i = f % nx;
    const size_t o = (size_t)(jf * nx + i);
    lo_face_interior_grp<WPF>(P, B, 1, (jf - 1) * nx + i, jf * nx + i, dt, B.fyh + o * nv, B.fyb + o * nv,
                              B.fyw + o * 4, sH[w], xch);
}

template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX) k_lo_walls(LoParams P, LoBuffers B) {
    if (eval_cached(B)) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    const double dt = B.dt[0];
    const int nx = P.nx, ny = P.ny, nv = P.nvel;
    const int f = blockIdx.x;
    const int side = f < nx ? -1 : 1, i = f % nx;
    const size_t o = (size_t)((side < 0 ? 0 : ny) * nx + i);
    lo_face_wall<VPT>(P, B, side, i, dt, B.fyh + o * nv, B.fyb + o * nv, B.fyw + o * 4,
                      B.wall_aero + ((side < 0 ? 0 : 1) * nx + i) * 3, red, rout);
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
    double acc[14];
#pragma unroll
    for (int m = 0; m < 13; ++m) acc[m] = 0.0;
    acc[13] = -INFINITY;   // max of -dt_local == -min(dt_local)
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        if (write_dt) acc[13] = fmax(acc[13], -__ldcg(B.dtl + c));
        if (write_diag) {
#pragma unroll
            for (int m = 0; m < 9; ++m) acc[m] += __ldcg(B.cell_diag + (size_t)c * kNDiag + m);
#pragma unroll
            for (int m = 0; m < 4; ++m) acc[9 + m] = fmax(acc[9 + m], __ldcg(B.cell_diag + (size_t)c * kNDiag + 9 + m));
        }
    }
    block_reduce<9, 5>(acc, red, rout);
    if (threadIdx.x == 0) {
        if (write_diag) {
            for (int m = 0; m < 13; ++m) B.diag[m] = acc[m];
        }
        if (write_dt) {
            B.dt[1] = B.dt[0];   // dt_global of the step that just completed
            B.dt[0] = P.fixed_dt > 0.0 ? P.fixed_dt : -acc[13];
        }
        *B.counter = 0u;
    }
}

__global__ void __launch_bounds__(256) k_lo_timestep(LoParams P, LoBuffers B) {
    if (halted(B)) return;
    __shared__ double red[8 * 64];
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
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_lo_cells(LoParams P, LoBuffers B) {
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    // per-cell scalars computed once (threads 0 and t1) and broadcast:
    //  [0..3] prim_old  [4] tau_old  [5] ok_old  [8..11] res_w  [12..15] prim_new  [16] tau_new  [17] ok_new
    //  [18..21] W_new  [22] dt_local(W_new)  [24..27] stream lambda  [28..31] old lambda  [32..35] new lambda
    //  [36..39] collision lambda  [40] projection flags
    __shared__ double sc[48];
    const int nv = P.nvel, tid = threadIdx.x, nx = P.nx;
    const int t1 = blockDim.x > 32 ? 32 : 0;   // a thread of the second warp, so the two solves overlap
    const int c = blockIdx.x, i = c % nx, j = c / nx;
    const double dt = B.dt[0];
    const double* hc = B.h + (size_t)c * nv;
    const double* bc = B.b + (size_t)c * nv;
    double h[VPT], b[VPT], rh[VPT], rb[VPT];
    double acc[28];
    const size_t fl = (size_t)(j * nx + i), fr = (size_t)(j * nx + wrapx(i + 1, nx));
    const size_t gl = (size_t)(j * nx + i), gr = (size_t)((j + 1) * nx + i);
    if (tid == 0) {
        const double* Wo = B.W + c * 4;
        Prim po;
        double to = 1.0;
        bool ok = get_primary(P.gm1, Wo, po);
        ok = ok && get_tau(P.mu_ref, P.omega, po, to);
        if (!ok) { po.r = 1.0; po.U = po.V = 0.0; po.L = 1.0; to = 1.0; }
        sc[0] = po.r; sc[1] = po.U; sc[2] = po.V; sc[3] = po.L; sc[4] = to; sc[5] = ok ? 1.0 : 0.0;
    }
    if (tid == t1) {
        double resw[4], Wn[4];
        if (MODE & MODE_RESIDUAL) {
            // AssembleMacroResidual (mod_Residual.f90:30-54)
#pragma unroll
            for (int m = 0; m < 4; ++m)
                resw[m] = (B.fxw[fl * 4 + m] - B.fxw[fr * 4 + m] + B.fyw[gl * 4 + m] - B.fyw[gr * 4 + m]) / P.area;
        } else {
#pragma unroll
            for (int m = 0; m < 4; ++m) resw[m] = B.res_w[c * 4 + m];
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) { Wn[m] = B.W[c * 4 + m] + resw[m]; sc[8 + m] = resw[m]; sc[18 + m] = Wn[m]; }
        if (MODE & MODE_UPDATE) {
            Prim pn;
            double tn = 1.0;
            bool ok = get_primary(P.gm1, Wn, pn);
            ok = ok && get_tau(P.mu_ref, P.omega, pn, tn);
            if (!ok) { pn.r = 1.0; pn.U = pn.V = 0.0; pn.L = 1.0; tn = 1.0; }
            sc[12] = pn.r; sc[13] = pn.U; sc[14] = pn.V; sc[15] = pn.L; sc[16] = tn; sc[17] = ok ? 1.0 : 0.0;
            bool dok;
            sc[22] = cell_dt(P, Wn, dok);
        }
    }
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        h[r] = hc[s.kk];
        b[r] = bc[s.kk];
    }
    if (MODE & MODE_RESIDUAL) {
        // AssembleMicroFluxResidual (mod_Residual.f90:60-76) and stream_h = res/dt (:81-95)
        const double area_inv = 1.0 / P.area;
        const double dti = 1.0 / dt;
#pragma unroll
        for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const int k = s.kk;
            const double wk = s.ok ? B.w[k] : 0.0;
            const double sh = (B.fxh[fl * nv + k] - B.fxh[fr * nv + k] + B.fyh[gl * nv + k] - B.fyh[gr * nv + k]) * area_inv;
            const double sb = (B.fxb[fl * nv + k] - B.fxb[fr * nv + k] + B.fyb[gl * nv + k] - B.fyb[gr * nv + k]) * area_inv;
            rh[r] = sh * dti;
            rb[r] = sb * dti;
            moment_add(wk, B.u[k], B.v[k], rh[r], rb[r], acc);
            acc[4] = fmax(acc[4], s.ok ? fabs(h[r]) : 0.0);
            acc[5] = fmax(acc[5], s.ok ? fabs(b[r]) : 0.0);
        }
        block_reduce<4, 2>(acc, red, rout);
        // EnforceStreamingMomentCompatibility (mod_ImplicitMicro.f90:293-306): stream onto rate_w
        double mom[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) mom[m] = acc[m];
        const double sh_ = fmax(acc[4], 1.0), sb_ = fmax(acc[5], 1.0);
#pragma unroll
        for (int m = 0; m < 10; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double wk = s.ok ? B.w[s.kk] : 0.0;
            gram_add(wk, fmax(fabs(h[r]), kEps * sh_), fmax(fabs(b[r]), kEps * sb_), B.u[s.kk], B.v[s.kk], acc);
        }
        block_reduce_smem<10, 0>(acc, red, rout);
        if (tid == 0) {
            double rhs[4], gm[16], lam[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) rhs[m] = sc[8 + m] * dti - mom[m];
            gram_expand(rout, gm);
            const bool pok = solve_dense4(gm, rhs, lam);
#pragma unroll
            for (int m = 0; m < 4; ++m) sc[24 + m] = pok ? lam[m] : 0.0;
            sc[40] = pok ? 0.0 : 1.0;
        }
        __syncthreads();
        double lam[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) lam[m] = sc[24 + m];
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
            const double e = 0.5 * (uk * uk + vk * vk);
            rh[r] = rh[r] + fmax(fabs(h[r]), kEps * sh_) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
            rb[r] = rb[r] + 0.5 * fmax(fabs(b[r]), kEps * sb_) * lam[3];
            moment_add(wk, uk, vk, rh[r], rb[r], acc);
            rh[r] = rh[r] * dt;   // res_h_flux_store = stream_h * dt (mod_Residual.f90:114-115)
            rb[r] = rb[r] * dt;
        }
        block_reduce_smem<4, 0>(acc, red, rout);
        if (tid == 0) {
            double rate[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) rate[m] = sc[8 + m] * dti;
            const double rs = fmax(fmax(fmax(fabs(rate[0]), fabs(rate[1])), fmax(fabs(rate[2]), fabs(rate[3]))), 1.0);
            double err = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) err = fmax(err, fabs(rout[m] - rate[m]));
            if (sc[40] != 0.0 || !(err <= 1.0e-10 * rs)) set_status(B.status, ST_PROJECTION);
        }
        if (MODE == MODE_RESIDUAL) {
#pragma unroll
            for (int r = 0; r < VPT; ++r) {
                const Slot s = slot(r, nv);
                if (!s.ok) continue;
                B.res_h[(size_t)c * nv + s.k] = rh[r];
                B.res_b[(size_t)c * nv + s.k] = rb[r];
            }
            if (tid < 4) B.res_w[c * 4 + tid] = sc[8 + tid];
        }
    } else {
        __syncthreads();   // the scalars written above
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            rh[r] = B.res_h[(size_t)c * nv + s.kk];
            rb[r] = B.res_b[(size_t)c * nv + s.kk];
        }
    }

    if (MODE == MODE_RESIDUAL && COLLISION) {
        // physical equilibrium and collision (mod_Residual.f90:116-127)
        const Prim p{sc[0], sc[1], sc[2], sc[3]};
        const double tau = sc[4];
        if (tid == 0 && sc[5] == 0.0) set_status(B.status, ST_GETPRIMARY);
        acc[0] = acc[1] = 0.0;
#pragma unroll
        for (int r = 0; r < VPT; ++r) {
            const Slot s = slot(r, nv);
            const double wk = s.ok ? B.w[s.kk] : 0.0;
            const double dvn = B.u[s.kk] - p.U, dvt = B.v[s.kk] - p.V, v2 = dvn * dvn + dvt * dvt;
            const double t = 0.5 * wk * (v2 * h[r] + b[r]);
            acc[0] += t * dvn;
            acc[1] += t * dvt;
        }
        block_reduce<2, 0>(acc, red, rout);
        const double q0 = acc[0], q1 = acc[1];
        double E[VPT], F[VPT];
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
            double rhs[4], gm[16], lam[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) rhs[m] = B.W[c * 4 + m] - rout[m];
            gram_expand(rout + 4, gm);
            const bool pok = solve_dense4(gm, rhs, lam);
#pragma unroll
            for (int m = 0; m < 4; ++m) sc[36 + m] = pok ? lam[m] : 0.0;
            if (!pok) set_status(B.status, ST_PROJECTION);
        }
        __syncthreads();
        double lam[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) lam[m] = sc[36 + m];
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
                B.peq_h[(size_t)c * nv + s.k] = Ep;
                B.peq_b[(size_t)c * nv + s.k] = Fp;
                B.pcol_h[(size_t)c * nv + s.k] = (Ep - h[r]) / tau;
                B.pcol_b[(size_t)c * nv + s.k] = (Fp - b[r]) / tau;
            }
        }
        block_reduce_smem<4, 0>(acc, red, rout);
        if (tid == 0) {
            const double* Wo = B.W + c * 4;
            const double rs = fmax(fmax(fmax(fabs(Wo[0]), fabs(Wo[1])), fmax(fabs(Wo[2]), fabs(Wo[3]))), 1.0);
            double err = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) err = fmax(err, fabs(rout[m] - Wo[m]));
            if (!(err <= 1.0e-10 * rs)) set_status(B.status, ST_PROJECTION);
        }
    }
    if (!(MODE & MODE_UPDATE)) return;

    // ---- ApplyExplicitUpdate (mod_TimeIntegrator.f90:16-134, 235-293)
    const Prim po{sc[0], sc[1], sc[2], sc[3]}, pn{sc[12], sc[13], sc[14], sc[15]};
    const double to = sc[4], tn = sc[16];
    if (tid == 0 && (sc[5] == 0.0 || sc[17] == 0.0)) set_status(B.status, ST_GETPRIMARY);
    // heat flux of the old state (GetHeatFlux_Vec with prim_old)
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        const double dvn = B.u[s.kk] - po.U, dvt = B.v[s.kk] - po.V, v2 = dvn * dvn + dvt * dvt;
        const double t = 0.5 * wk * (v2 * h[r] + b[r]);
        acc[0] += t * dvn;
        acc[1] += t * dvt;
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
            const Slot s = slot(r, nv);
            const double uk = B.u[s.kk], vk = B.v[s.kk];
            double dvn = uk - po.U, dvt = vk - po.V, v2 = dvn * dvn + dvt * dvt;
            double H = pro * exp(-po.L * v2), Bm = H * bfo, qd = dvn * q0 + dvt * q1, sH = 2.0 * po.L * v2 - 4.0;
            Ho[r] = H + co * qd * sH * H;
            Bo[r] = Bm + co * qd * (sH + c2ck) * Bm;
            dvn = uk - pn.U; dvt = vk - pn.V; v2 = dvn * dvn + dvt * dvt;
            H = prn * exp(-pn.L * v2); Bm = H * bfn; qd = dvn * q0 + dvt * q1; sH = 2.0 * pn.L * v2 - 4.0;
            Hn[r] = H + cn * qd * sH * H;
            Bn[r] = Bm + cn * qd * (sH + c2ck) * Bm;
            acc[0] = fmax(acc[0], s.ok ? fabs(Ho[r]) : 0.0);
            acc[1] = fmax(acc[1], s.ok ? fabs(Bo[r]) : 0.0);
            acc[2] = fmax(acc[2], s.ok ? fabs(Hn[r]) : 0.0);
            acc[3] = fmax(acc[3], s.ok ? fabs(Bn[r]) : 0.0);
        }
        block_reduce<0, 4>(acc, red, rout);
    }
    const double sHo = fmax(acc[0], 1.0), sBo = fmax(acc[1], 1.0), sHn = fmax(acc[2], 1.0), sBn = fmax(acc[3], 1.0);
#pragma unroll
    for (int m = 0; m < 28; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        moment_add(wk, uk, vk, Ho[r], Bo[r], acc);
        gram_add(wk, fmax(fabs(Ho[r]), kEps * sHo), fmax(fabs(Bo[r]), kEps * sBo), uk, vk, acc + 4);
        moment_add(wk, uk, vk, Hn[r], Bn[r], acc + 14);
        gram_add(wk, fmax(fabs(Hn[r]), kEps * sHn), fmax(fabs(Bn[r]), kEps * sBn), uk, vk, acc + 18);
    }
    block_reduce_smem<28, 0>(acc, red, rout);
    // two ProjectToConservedMoments solves (mod_TimeIntegrator.f90:267-274), one per warp
    if (tid == 0) {
        double to4[4], rhs[4], gm[16], l[4];
        get_conserved(P.gm1, po, to4);
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = to4[m] - rout[m];
        gram_expand(rout + 4, gm);
        const bool ok = solve_dense4(gm, rhs, l);
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[28 + m] = ok ? l[m] : 0.0;
        if (!ok) set_status(B.status, ST_PROJECTION);
    }
    if (tid == t1) {
        double rhs[4], gm[16], l[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) rhs[m] = sc[18 + m] - rout[14 + m];
        gram_expand(rout + 18, gm);
        const bool ok = solve_dense4(gm, rhs, l);
#pragma unroll
        for (int m = 0; m < 4; ++m) sc[32 + m] = ok ? l[m] : 0.0;
        if (!ok) set_status(B.status, ST_PROJECTION);
    }
    __syncthreads();
    double lo[4], ln[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) { lo[m] = sc[28 + m]; ln[m] = sc[32 + m]; }
    const double inv = 1.0 / (1.0 + 0.5 * dt / tn);
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0, e = 0.5 * (uk * uk + vk * vk);
        const double Hop = Ho[r] + fmax(fabs(Ho[r]), kEps * sHo) * (lo[0] + uk * lo[1] + vk * lo[2] + e * lo[3]);
        const double Bop = Bo[r] + 0.5 * fmax(fabs(Bo[r]), kEps * sBo) * lo[3];
        const double Hnp = Hn[r] + fmax(fabs(Hn[r]), kEps * sHn) * (ln[0] + uk * ln[1] + vk * ln[2] + e * ln[3]);
        const double Bnp = Bn[r] + 0.5 * fmax(fabs(Bn[r]), kEps * sBn) * ln[3];
        moment_add(wk, uk, vk, Hop, Bop, acc);
        moment_add(wk, uk, vk, Hnp, Bnp, acc + 4);
        const double hnew = (h[r] + rh[r] + 0.5 * dt * (Hnp / tn + (Hop - h[r]) / to)) * inv;
        const double bnew = (b[r] + rb[r] + 0.5 * dt * (Bnp / tn + (Bop - b[r]) / to)) * inv;
        if (s.ok) {
            B.h[(size_t)c * nv + s.k] = hnew;
            B.b[(size_t)c * nv + s.k] = bnew;
        }
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    if (tid == 0) {
        double to4[4], Wn[4], Wold[4];
        get_conserved(P.gm1, po, to4);
#pragma unroll
        for (int m = 0; m < 4; ++m) { Wn[m] = sc[18 + m]; Wold[m] = B.W[c * 4 + m]; }
        const double ro = fmax(fmax(fmax(fabs(to4[0]), fabs(to4[1])), fmax(fabs(to4[2]), fabs(to4[3]))), 1.0);
        const double rn = fmax(fmax(fmax(fabs(Wn[0]), fabs(Wn[1])), fmax(fabs(Wn[2]), fabs(Wn[3]))), 1.0);
        double eo = 0.0, en = 0.0;
        for (int m = 0; m < 4; ++m) { eo = fmax(eo, fabs(rout[m] - to4[m])); en = fmax(en, fabs(rout[4 + m] - Wn[m])); }
        if (!(eo <= 1.0e-10 * ro) || !(en <= 1.0e-10 * rn)) set_status(B.status, ST_PROJECTION);
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
        B.dtl[c] = sc[22];
    }
    last_cta_epilogue(P, B, true, true, red, rout);
}

// -------------------------------------------------------------------------------------------
// InitFlow_Freestream (mod_InitializeFlow.f90:826-856) + the cold-start moment projection
// EnforceAcceptedMomentCompatibility (mod_ImplicitMicro.f90, via InitializeSteadyImplicit).
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX) k_lo_init(LoParams P, LoBuffers B, double rho, double U, double V,
                                                   double tn) {
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, tid = threadIdx.x, c = blockIdx.x;
    const Prim p{rho, U, V, 1.0 / tn};
    double W[4];
    get_conserved(P.gm1, p, W);
    const double pref = p.r * (p.L / kPi), bfac = (double)P.ck / (2.0 * p.L);
    double H[VPT], Bm[VPT], acc[14];
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double dvn = B.u[s.kk] - p.U, dvt = B.v[s.kk] - p.V;
        H[r] = pref * exp(-p.L * (dvn * dvn + dvt * dvt));
        Bm[r] = H[r] * bfac;
        acc[0] = fmax(acc[0], s.ok ? fabs(H[r]) : 0.0);
        acc[1] = fmax(acc[1], s.ok ? fabs(Bm[r]) : 0.0);
    }
    block_reduce<0, 2>(acc, red, rout);
    const double sh = fmax(acc[0], 1.0), sb = fmax(acc[1], 1.0);
#pragma unroll
    for (int m = 0; m < 14; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        moment_add(wk, B.u[s.kk], B.v[s.kk], H[r], Bm[r], acc);
        gram_add(wk, fmax(fabs(H[r]), kEps * sh), fmax(fabs(Bm[r]), kEps * sb), B.u[s.kk], B.v[s.kk], acc + 4);
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
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const double uk = B.u[s.k], vk = B.v[s.k], e = 0.5 * (uk * uk + vk * vk);
        B.h[(size_t)c * nv + s.k] = H[r] + fmax(fabs(H[r]), kEps * sh) * (lam[0] + uk * lam[1] + vk * lam[2] + e * lam[3]);
        B.b[(size_t)c * nv + s.k] = Bm[r] + 0.5 * fmax(fabs(Bm[r]), kEps * sb) * lam[3];
    }
    if (tid < 4) B.W[c * 4 + tid] = W[tid];
}

// -------------------------------------------------------------------------------------------
// Host-visible launchers (used by ugks_capi.cu).  Tile = (velocities per thread, threads):
// nvel <= 1024 -> (4, <=256 threads); nvel <= 2560 -> (5, <=512 threads).
int lo_vpt(int nvel) { return nvel <= 4 * 256 ? 4 : 5; }

int lo_threads(int nvel) {
    const int vpt = lo_vpt(nvel);
    int t = (nvel + vpt - 1) / vpt;
    t = (t + 31) / 32 * 32;
    return t < 32 ? 32 : t;
}

cudaError_t launch_lo_slopes(const LoParams& P, const LoBuffers& B, cudaStream_t s) {
    const dim3 grid((unsigned)((P.nvel + 255) / 256), (unsigned)(P.nx * P.ny));
    k_lo_slopes<<<grid, 256, 0, s>>>(P, B);
    return cudaGetLastError();
}

cudaError_t launch_lo_faces(const LoParams& P, const LoBuffers& B, cudaStream_t s) {
    const int nface = P.nx * P.ny + P.nx * (P.ny - 1);
    const int nt = lo_threads(P.nvel);
    if (P.nvel <= 1024) k_lo_faces_grp<4, 1><<<(unsigned)((nface + 3) / 4), 128, 0, s>>>(P, B);
    else if (lo_vpt(P.nvel) == 4) k_lo_faces<4, 256><<<nface, nt, 0, s>>>(P, B);
    else k_lo_faces<5, 512><<<nface, nt, 0, s>>>(P, B);
    return cudaGetLastError();
}

cudaError_t launch_lo_walls(const LoParams& P, const LoBuffers& B, cudaStream_t s) {
    const int nt = lo_threads(P.nvel);
    if (lo_vpt(P.nvel) == 4) k_lo_walls<4, 256><<<2 * P.nx, nt, 0, s>>>(P, B);
    else k_lo_walls<5, 512><<<2 * P.nx, nt, 0, s>>>(P, B);
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

// -------------------------------------------------------------------------------------------
// Steady output fields of one cell (Output, mod_Output.f90:102-116): r, u, v, T = 1/lambda,
// p = r T / 2, the stress tensor sxx, sxy, syy (Get_Stress_Vec with GetPressure_Vec,
// mod_Tools.f90:326-347,409-432) and the heat flux qx, qy (GetHeatFlux_Vec, mod_Tools.f90:355-373).
template <int VPT, int NTMAX>
__global__ void __launch_bounds__(NTMAX, 512 / NTMAX) k_lo_macro_fields(LoParams P, LoBuffers B, double* out) {
    __shared__ double red[8 * 64];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, c = blockIdx.x;
    double w4[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) w4[m] = B.W[c * 4 + m];
    Prim p;
    const bool ok = get_primary(P.gm1, w4, p);
    if (!ok) { p.r = 1.0; p.U = p.V = 0.0; p.L = 1.0; }
    double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const double wk = s.ok ? B.w[s.kk] : 0.0;
        const double dvn = B.u[s.kk] - p.U, dvt = B.v[s.kk] - p.V, v2 = dvn * dvn + dvt * dvt;
        const double h = B.h[(size_t)c * nv + s.kk], b = B.b[(size_t)c * nv + s.kk];
        acc[0] += wk * v2 * h;                       // energy_sum
        acc[1] += wk * b;                            // b_sum
        acc[2] += wk * dvn * dvn * h;
        acc[3] += wk * dvn * dvt * h;
        acc[4] += wk * dvt * dvt * h;
        acc[5] += 0.5 * wk * dvn * (v2 * h + b);
        acc[6] += 0.5 * wk * dvt * (v2 * h + b);
    }
    block_reduce_smem<7, 0>(acc, red, rout);
    if (threadIdx.x == 0) {
        const double pr = (rout[0] + rout[1]) / ((double)P.ck + 2.0);
        const double T = 1.0 / p.L;
        double* o = out + (size_t)c * 10;
        o[0] = p.r; o[1] = p.U; o[2] = p.V; o[3] = T; o[4] = 0.5 * p.r * T;
        o[5] = rout[2] - pr; o[6] = rout[3]; o[7] = rout[4] - pr;
        o[8] = rout[5]; o[9] = rout[6];
        if (!ok) set_status(B.status, ST_GETPRIMARY);
    }
}

cudaError_t launch_lo_macro_fields(const LoParams& P, const LoBuffers& B, double* out, cudaStream_t s) {
    if (lo_vpt(P.nvel) == 4) k_lo_macro_fields<4, 256><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, out);
    else k_lo_macro_fields<5, 512><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, out);
    return cudaGetLastError();
}

cudaError_t launch_lo_init(const LoParams& P, const LoBuffers& B, double rho, double U, double V, double tn,
                           cudaStream_t s) {
    if (lo_vpt(P.nvel) == 4) k_lo_init<4, 256><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, rho, U, V, tn);
    else k_lo_init<5, 512><<<P.nx * P.ny, lo_threads(P.nvel), 0, s>>>(P, B, rho, U, V, tn);
    return cudaGetLastError();
}

}  // namespace ugks
