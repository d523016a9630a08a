// ugks_s2_adjoint.cu -- reverse-mode (adjoint) kernels of the S2CN2 step on sm_100a (FP64).
//
// One step of ugks_s2cn2.cu is TimeStep, the S2 evaluation with the accepted state's targets,
// k_cn_stream, the targets of the stream state and k_cn_collide.  Its adjoint runs the same stages
// backwards, each kernel the transpose of the forward kernel's map, after a forward re-run of the step
// has refilled the evaluation scratch:
//   k_adj_collide      : the CN collision (mod_S2D1.f90:1376-1421): 2x2 heat-flux solve, h_new.
//   k_adj_targets      : build_targets of the stream state (mod_S2D1.f90:1246-1300): the Gauss-weighted
//                        sums, make_mke (mod_S2D1.f90:111-151) and the discrete closure of each volume
//                        node (solve_q_first, mod_CorrectedWF2DClosure.f90:331-426) by the
//                        implicit-function theorem: d theta = J^-1 d W at the converged closure.
//   k_adj_macro_cells  : the mean-shifted volume node states (s2d1_cell9 + mean shift) of the stream state.
//   k_adj_stream       : the stream state, the residual and the CN right-hand side.
//   k_adj_face_nodes   : ugks_node (mod_S2D1.f90:421-521) at one interior face Gauss node per warp,
//                        flux and node scalars together (closure, directions, time coefficients).
//   k_adj_wall_nodes   : the multiscale wall node (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184) and
//                        the wall outputs (PublishWallDiagnostics, mod_S2NativeAdapter.f90:1075-1097).
//   k_adj_macro_faces  : the macro WENO slopes of W at the interior faces.
//   k_adj_recon2/1     : the second-layer templates with the positivity limiter (limit_cell_outputs,
//                        mod_S2D1.f90:315-345) and the first-layer WENO-AO (mod_S2D1Reconstruction.f90).
//
// The time step is constant along the trajectory (the velocity table's extent sets it; k_adj_stream
// checks that on every state and raises ST_ADJOINT_DT otherwise).  The velocity-independent scalar
// chains (tau and the time coefficients, the primitive variables, the wall state, its micro slopes and
// erfc moments) are differentiated in forward mode with one input direction per warp lane (Dl below)
// and transposed; every per-velocity expression is transposed by hand.  Scatter-adjoints into the
// state, the first layer and W accumulate with atomicAdd (one ulp of ordering noise run to run).
#include "ugks_s2_adjoint.cuh"
#include "ugks_s2_math.cuh"

namespace ugks {
namespace {


// ---------------------------------------------------------------------------------------------
// forward mode on one input direction per lane (the double versions of the math functions stay visible
// beside the Dl overloads)
using ::erfc;
using ::exp;
using ::pow;
using ::sqrt;
struct Dl {
    double v, d;
};
__device__ __forceinline__ Dl operator+(Dl a, Dl b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dl operator-(Dl a, Dl b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dl operator*(Dl a, Dl b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dl operator/(Dl a, Dl b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dl operator-(Dl a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dl operator+(Dl a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dl operator-(double a, Dl b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dl operator*(Dl a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dl operator*(double a, Dl b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dl operator/(Dl a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dl operator/(double a, Dl b) {
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dl exp(Dl a) {
    const double e = ::exp(a.v);
    return {e, e * a.d};
}
__device__ __forceinline__ Dl sqrt(Dl a) {
    const double s = ::sqrt(a.v);
    return {s, 0.5 * a.d / s};
}
// d erfc(x)/dx = -2/sqrt(pi) exp(-x^2)
__device__ __forceinline__ Dl erfc(Dl a) { return {::erfc(a.v), -1.1283791670955125739 * ::exp(-a.v * a.v) * a.d}; }
__device__ __forceinline__ Dl pow(Dl a, double e) {
    const double p = ::pow(a.v, e);
    return {p, e * ::pow(a.v, e - 1.0) * a.d};
}
__device__ __forceinline__ double val(Dl x) { return x.v; }

// lane l < n carries the direction of input l: x[i] = (in[i], i == lane)
template <int N>
__device__ __forceinline__ void seed_lane(const double in[N], Dl x[N]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = {in[i], i == lane ? 1.0 : 0.0};
}
// g_in[l] = sum_o g_out[o] d out[o] / d in[l] on lane l, gathered to every lane as gin[0..N)
template <int NO, int NI>
__device__ __forceinline__ void transpose_lanes(const Dl out[NO], const double gout[NO], double gin[NI]) {
    double s = 0.0;
#pragma unroll
    for (int o = 0; o < NO; ++o) s += gout[o] * out[o].d;
#pragma unroll
    for (int i = 0; i < NI; ++i) gin[i] = __shfl_sync(0xffffffffu, s, i);
}

// ---------------------------------------------------------------------------------------------
// scalar chains, generic over double / Dl, in the forward kernels' arithmetic

// s2_tau (mod_S2PhysicalGas.f90:9-20) with mu_ref as an input: GetTau of (rho, U, V, 0.5 rho / p)
template <class T>
__device__ __forceinline__ T tau_of(const LoParams& P, const T w[4], T mu) {
    const T pr = (2.0 / (double)(P.ck + 2)) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    const T L = 0.5 * w[0] / pr;
    const T muv = mu * pow(1.0 / L, P.omega);
    return muv / (0.5 * w[0] / L);
}

// [tau, ux, vy] of a cell state (k_cn_stream / k_cn_collide: s2_tau and s2_primitive)
template <class T>
__device__ __forceinline__ void cell_chain(const LoParams& P, const T w[4], T mu, T out[3]) {
    out[0] = tau_of(P, w, mu);
    out[1] = w[1] / w[0];
    out[2] = w[2] / w[0];
}

// make_mke's primitive scalars (ux, vy, lam, coeff) of a node state (w_make_mke)
template <class T>
__device__ __forceinline__ void mke_chain(const LoParams& P, const T w[4], T out[4]) {
    const T ux = w[1] / w[0], vy = w[2] / w[0];
    const T eint = w[3] - 0.5 * w[0] * (ux * ux + vy * vy);
    const T th = (2.0 / (double)(P.ck + 2)) * eint / w[0];
    const T lam = 0.5 / th;
    out[0] = ux;
    out[1] = vy;
    out[2] = lam;
    out[3] = 0.8 * (1.0 - P.pr) * lam * lam / w[0];
}

// ugks_node's W0 scalars (k_s2_face_nodes): Mt of tau(W0), make_mke's primitive scalars, and the
// analytic Maxwellian's (rho, u, v, T) used by q0
template <class T>
__device__ __forceinline__ void face_chain(const LoParams& P, double dt, const T w[4], T mu, T out[13]) {
    const T tau = tau_of(P, w, mu);
    const T ex = exp((-dt) / tau);
    const T m3 = tau * (1.0 - ex);
    const T m4 = -tau * dt * ex + tau * m3;
    const T m0 = dt - m3;
    out[0] = m0;
    out[1] = -tau * m0 + m4;
    out[2] = 0.5 * dt * dt - tau * m0;
    out[3] = m3;
    out[4] = m4;
    mke_chain(P, w, out + 5);
    const T nu = w[1] / w[0], nvv = w[2] / w[0];
    out[9] = w[0];
    out[10] = nu;
    out[11] = nvv;
    out[12] = 4.0 * (w[3] / w[0] - 0.5 * (nu * nu + nvv * nvv)) / (double)(P.ck + 2);
}

// ---------------------------------------------------------------------------------------------
// per-velocity closure pieces
struct QV {
    double qh, qb, ld[4], ldb[4], du, dv, c2;
};
__device__ __forceinline__ QV qv_at(const S2Th& t, double u, double v) {
    QV q;
    const S2Q s = s2_q(t, u, v);
    q.qh = s.qh;
    q.qb = s.qb;
#pragma unroll
    for (int a = 0; a < 4; ++a) { q.ld[a] = s.ld[a]; q.ldb[a] = s.ldb[a]; }
    q.du = u - t.u;
    q.dv = v - t.v;
    q.c2 = q.du * q.du + q.dv * q.dv;
    return q;
}
// out[b] = sum_a V[a] d(q ld_a)/d theta_b for the h field (hb = 0) or the b field (hb = 1):
// d(q ld_a)/d theta_b = q (ld_a ld_b + d ld_a / d theta_b), theta = (rho, u, v, T_native)
__device__ __forceinline__ void vhess(const S2Th& t, const QV& q, int hb, const double V[4], double out[4]) {
    const double* ld = hb ? q.ldb : q.ld;
    const double qq = hb ? q.qb : q.qh;
    const double it = t.itw, it2 = it * it;
    const double s = V[0] * ld[0] + V[1] * ld[1] + V[2] * ld[2] + V[3] * ld[3];
    out[0] = qq * (s * ld[0] - V[0] * t.ir * t.ir);
    out[1] = qq * (s * ld[1] - 2.0 * V[1] * it - 2.0 * q.du * V[3] * it2);
    out[2] = qq * (s * ld[2] - 2.0 * V[2] * it - 2.0 * q.dv * V[3] * it2);
    const double d33 = hb ? -2.0 * q.c2 * it2 * it : it2 - 2.0 * q.c2 * it2 * it;
    out[3] = qq * (s * ld[3] - 2.0 * q.du * V[1] * it2 - 2.0 * q.dv * V[2] * it2 + V[3] * d33);
}
// cotangent of (fh, fb) from the cotangent g of their moments [sum w fh, sum w u fh, sum w v fh,
// sum w (|c|^2 fh + fb) / 2]
__device__ __forceinline__ double psi_h(double w, double u, double v, const double g[4]) {
    return w * (g[0] + u * g[1] + v * g[2] + 0.5 * (u * u + v * v) * g[3]);
}
__device__ __forceinline__ double psi_b(double w, const double g[4]) { return 0.5 * w * g[3]; }

// x = J^-T g with J row-major
__device__ __forceinline__ bool solve_t4(const double* jac, const double g[4], double x[4]) {
    double jt[16];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) jt[r * 4 + c] = jac[c * 4 + r];
    return s2_solve4(jt, g, x);
}

// d heat / d (ux, vy) of one velocity with (fh, fb) = the heat's argument, cotangents (gx, gy)
__device__ __forceinline__ void heat_shift_adj(double w, double cx, double cy, double fh, double fb, double gx,
                                               double gy, double& gux, double& gvy) {
    const double c2 = cx * cx + cy * cy, base = c2 * fh + fb, xy = w * cx * cy * fh;
    gux += gx * (0.5 * w * (-base - 2.0 * cx * cx * fh)) - gy * xy;
    gvy += -gx * xy + gy * (0.5 * w * (-base - 2.0 * cy * cy * fh));
}

// ---------------------------------------------------------------------------------------------
// WENO-AO(5,3) weights: the transpose of fw(q) (weno_coefficients, mod_S2D1Reconstruction.f90:168-204),
// from the forward's intermediates x (s2_weno_x): only products, the forward holds the reciprocals.
//   fw_3 = alpha_3 isa / 0.85, fw_c = alpha_c isa - gam_c fw_3 (c < 3), isa = 1 / sum(alpha),
//   alpha_c = gam_c (1 + r_c^2), r_c = tau inv_c, inv_c = 1 / (beta_c + 1e-8), tau = mean |beta_3 - beta_c|
__device__ void weno_weights_vjp(const S2Weno& w, const S2WenoX& x, const double gfw[4], double gq[5]) {
    const double q1 = w.q[0], q2 = w.q[1], q3 = w.q[2], q4 = w.q[3], q5 = w.q[4];
    const double t0 = q1 - 2 * q2 + q3, u0 = q1 - 4 * q2 + 3 * q3;
    const double t1 = q2 - 2 * q3 + q4, u1 = q2 - q4;
    const double t2 = q3 - 2 * q4 + q5, u2 = 3 * q3 - 4 * q4 + q5;
    const double gam[4] = {0.01125, 0.1275, 0.01125, 0.85};
    double alpha[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) alpha[c] = gam[c] * (1.0 + x.r[c] * x.r[c]);
    const double g3 = gfw[3] - (gam[0] * gfw[0] + gam[1] * gfw[1] + gam[2] * gfw[2]);
    const double g3s = g3 * (1.0 / 0.85);
    const double common = (gfw[0] * alpha[0] + gfw[1] * alpha[1] + gfw[2] * alpha[2] + g3s * alpha[3]) * (x.isa * x.isa);
    double ga[4];
    ga[0] = gfw[0] * x.isa - common;
    ga[1] = gfw[1] * x.isa - common;
    ga[2] = gfw[2] * x.isa - common;
    ga[3] = g3s * x.isa - common;
    double gtau = 0.0, gb[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double gr = ga[c] * gam[c] * 2.0 * x.r[c];
        gtau += gr * x.inv[c];
        gb[c] = -gr * x.r[c] * x.inv[c];
    }
    // tau = mean |beta_3 - beta_c|
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double gt = gtau * (1.0 / 3.0) * x.sg[c];
        gb[3] += gt;
        gb[c] -= gt;
    }
    // beta_c(q)
    const double a0 = 13.0 / 6.0 * t0 * gb[0], b0 = 0.5 * u0 * gb[0];
    const double a1 = 13.0 / 6.0 * t1 * gb[1], b1 = 0.5 * u1 * gb[1];
    const double a2 = 13.0 / 6.0 * t2 * gb[2], b2 = 0.5 * u2 * gb[2];
    const double g5 = gb[3] * (1.0 / 5040.0);
    gq[0] += a0 + b0 + g5 * (13816.0 * q1 - 38947.0 * q4 - 51001.0 * q2 + 67923.0 * q3 + 8209.0 * q5);
    gq[1] += -2.0 * a0 - 4.0 * b0 + a1 + b1 +
             g5 * (209926.0 * q2 - 51001.0 * q1 + 179098.0 * q4 - 38947.0 * q5 - 299076.0 * q3);
    gq[2] += a0 + 3.0 * b0 - 2.0 * a1 + a2 + 3.0 * b2 +
             g5 * (462306.0 * q3 - 299076.0 * q2 + 67923.0 * q1 - 299076.0 * q4 + 67923.0 * q5);
    gq[3] += a1 - b1 - 2.0 * a2 - 4.0 * b2 +
             g5 * (-38947.0 * q1 + 209926.0 * q4 + 179098.0 * q2 - 299076.0 * q3 - 51001.0 * q5);
    gq[4] += a2 + b2 + g5 * (-38947.0 * q2 + 67923.0 * q3 + 8209.0 * q1 - 51001.0 * q4 + 13816.0 * q5);
}

// transpose of r = sum_c fw[c] sum_k T[c][k] v[k] (s2_cand_sum) with cotangent g: gv and gfw accumulate
__device__ __forceinline__ void cand_vjp(const double fw[4], const double v[5], const double (*T)[5], double g,
                                         double gv[5], double gfw[4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double cand = 0.0;
        const double gf = g * fw[c];
#pragma unroll
        for (int k = (c < 3 ? c : 0); k <= (c < 3 ? c + 2 : 4); ++k) {
            cand = cand + T[c][k] * v[k];
            gv[k] += gf * T[c][k];
        }
        gfw[c] += g * cand;
    }
}

// transpose of the values (and derivatives) of the WENO-AO interpolant (w, x of s2_weno_x) at points pts[i]:
// gval[i], gder[i] the cotangents of the value and the xi-derivative at pts[i]; gq accumulates
template <int NP>
__device__ __forceinline__ void weno_points_vjp(const S2Weno& w, const S2WenoX& x, const int pts[NP],
                                                const double gval[NP], const double gder[NP], double gq[5]) {
    double gfw[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        if (gval[i] != 0.0) cand_vjp(w.fw, w.q, c_s2p.E[pts[i]], gval[i], gq, gfw);
        if (gder[i] != 0.0) cand_vjp(w.fw, w.q, c_s2p.D[pts[i]], gder[i], gq, gfw);
    }
    weno_weights_vjp(w, x, gfw, gq);
}
// the same from the stencil alone (the weights recomputed)
template <int NP>
__device__ __forceinline__ void weno_points_vjp(const double q[5], const int pts[NP], const double gval[NP],
                                                const double gder[NP], double gq[5]) {
    S2Weno w;
    S2WenoX x;
    s2_weno_x<true>(q, w, &x);
    weno_points_vjp<NP>(w, x, pts, gval, gder, gq);
}

// s2_companion3 with the weights' intermediates kept for companion3_vjp (the same values bit for bit)
__device__ __forceinline__ bool companion3_fwd(const double q[5], const double comp[5], double val[3], double der[3],
                                               double cval[3], S2Weno& w, S2WenoX& x) {
    if (!s2_weno_x<true>(q, w, &x)) return false;
    bool ok = true;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        s2_at(w, S2_G0 + s, val[s], der[s]);
        cval[s] = s2_cand_sum(w.fw, comp, c_s2p.E[S2_G0 + s]);
        ok = ok && isfinite(val[s]) && isfinite(der[s]) && isfinite(cval[s]);
    }
    return ok;
}

// transpose of companion_eval3 (s2_companion3): val[s], der[s] of the interpolant of q and cval[s] of the
// companion samples with q's weights, at the 3 Gauss nodes
__device__ __forceinline__ void companion3_vjp(const S2Weno& w, const S2WenoX& x, const double comp[5],
                                               const double gval[3], const double gder[3], const double gcval[3],
                                               double gq[5], double gcomp[5]) {
    double gfw[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        cand_vjp(w.fw, w.q, c_s2p.E[S2_G0 + s], gval[s], gq, gfw);
        cand_vjp(w.fw, w.q, c_s2p.D[S2_G0 + s], gder[s], gq, gfw);
        cand_vjp(w.fw, comp, c_s2p.E[S2_G0 + s], gcval[s], gcomp, gfw);
    }
    weno_weights_vjp(w, x, gfw, gq);
}
__device__ __forceinline__ void companion3_vjp(const double q[5], const double comp[5], const double gval[3],
                                               const double gder[3], const double gcval[3], double gq[5],
                                               double gcomp[5]) {
    S2Weno w;
    S2WenoX x;
    s2_weno_x<true>(q, w, &x);
    companion3_vjp(w, x, comp, gval, gder, gcval, gq, gcomp);
}

// transpose of s2_wall_eval (the one-sided quartic of the wall rows): cotangents of its value and
// derivative at xi into gq
__device__ __forceinline__ void wall_eval_vjp(int j, int ny, double xi, double gval, double gder, double gq[5]) {
    const int side = (j + 1 <= 3) ? 0 : 1, dist = side == 0 ? j : ny - 1 - j;
    double xp[5], dxp[5];
    xp[0] = 1.0;
    dxp[0] = 0.0;
#pragma unroll
    for (int d = 1; d < 5; ++d) { xp[d] = xp[d - 1] * xi; dxp[d] = (double)d * xp[d - 1]; }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < 5; ++d) s += c_s2.wall[side][dist][k][d] * (gval * xp[d] + gder * dxp[d]);
        gq[k] += s;
    }
}

__device__ __forceinline__ void atomic_add(double* p, double v) {
    if (v != 0.0) atomicAdd(p, v);
}

// ---------------------------------------------------------------------------------------------
// the CN collision (k_cn_collide): one CTA per cell
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_adj_collide(LoParams P, LoBuffers B, S2Buffers Tn, CnBuffers C, AdjBuffers A) {
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[24];   // [0] tau [1] ux [2] vy [3..17] d(tau, ux, vy)/d(wn, mu)
    const int nv = P.nvel, tid = threadIdx.x, c = blockIdx.x;
    const double dt = B.dt[0];
    const double* wn = C.ws + c * 4;
    if (tid < 32) {   // tau, ux, vy of the stream state and their Jacobian in (wn, mu_ref), one input per lane
        const double in[5] = {wn[0], wn[1], wn[2], wn[3], P.mu_ref};
        Dl x[5], o[3];
        seed_lane<5>(in, x);
        cell_chain(P, x, x[4], o);
        if (tid < 5)
#pragma unroll
            for (int q = 0; q < 3; ++q) sc[3 + q * 5 + tid] = o[q].d;
        if (tid == 0) { sc[0] = o[0].v; sc[1] = o[1].v; sc[2] = o[2].v; }
    }
    __syncthreads();
    const double tau = sc[0], ux = sc[1], vy = sc[2];
    const double beta = dt / (2.0 * tau), opb = 1.0 + beta;
    // the forward sums: heat of rh, M, K_x, K_y
    double acc[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0, cx = uk - ux, cy = vk - vy;
        const double c2 = cx * cx + cy * cy;
        const double hh[4] = {C.rh[q], Tn.mh[q], Tn.kxh[q], Tn.kyh[q]}, bb[4] = {C.rb[q], Tn.mb[q], Tn.kxb[q], Tn.kyb[q]};
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            acc[2 * f] += 0.5 * wk * cx * (c2 * hh[f] + bb[f]);
            acc[2 * f + 1] += 0.5 * wk * cy * (c2 * hh[f] + bb[f]);
        }
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    // a = I (1 + beta) - beta kappa, kappa(:, 1) = heat(K_x), kappa(:, 2) = heat(K_y); r = a^-1 (heat(rh) - heat(M))
    const double S0x = rout[0], S0y = rout[1], S1x = rout[2], S1y = rout[3];
    const double Kx0 = rout[4], Kx1 = rout[5], Ky0 = rout[6], Ky1 = rout[7];
    const double a11 = 1.0 + beta - beta * Kx0, a21 = -beta * Kx1, a12 = -beta * Ky0, a22 = 1.0 + beta - beta * Ky1;
    const double det = a11 * a22 - a12 * a21;
    const double rhs0 = S0x - S1x, rhs1 = S0y - S1y;
    const double r0 = (rhs0 * a22 - a12 * rhs1) / det, r1 = (a11 * rhs1 - rhs0 * a21) / det;
    // pass 1: cotangents of beta and r
#pragma unroll
    for (int m = 0; m < 3; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const size_t q = (size_t)c * nv + s.k;
        const double eqh = Tn.mh[q] + Tn.kxh[q] * r0 + Tn.kyh[q] * r1, eqb = Tn.mb[q] + Tn.kxb[q] * r0 + Tn.kyb[q] * r1;
        const double hn = (C.rh[q] + beta * eqh) / opb, bn = (C.rb[q] + beta * eqb) / opb;
        const double gh = A.gho[q], gb = A.gbo[q];
        const double geh = beta / opb * gh, geb = beta / opb * gb;
        acc[0] += (gh * (eqh - hn) + gb * (eqb - bn)) / opb;
        acc[1] += geh * Tn.kxh[q] + geb * Tn.kxb[q];
        acc[2] += geh * Tn.kyh[q] + geb * Tn.kyb[q];
    }
    block_reduce_smem<3, 0>(acc, red, rout);
    // the 2x2 solve: g_rhs = a^-T g_r, g_a = -g_rhs r^T
    const double gr0 = rout[1], gr1 = rout[2];
    const double grhs0 = (a22 * gr0 - a21 * gr1) / det, grhs1 = (-a12 * gr0 + a11 * gr1) / det;
    const double ga11 = -grhs0 * r0, ga12 = -grhs0 * r1, ga21 = -grhs1 * r0, ga22 = -grhs1 * r1;
    double gbeta = rout[0] + ga11 * (1.0 - Kx0) + ga12 * (-Ky0) + ga21 * (-Kx1) + ga22 * (1.0 - Ky1);
    // cotangents of the four heat sums (rh, M, K_x, K_y), x and y components
    const double gS[8] = {grhs0, grhs1, -grhs0, -grhs1, -beta * ga11, -beta * ga21, -beta * ga12, -beta * ga22};
    // pass 2: the per-velocity cotangents, and d/d(ux, vy) of the heat sums
    double gux = 0.0, gvy = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const size_t q = (size_t)c * nv + s.k;
        const double uk = B.u[s.k], vk = B.v[s.k], wk = B.w[s.k], cx = uk - ux, cy = vk - vy;
        const double c2 = cx * cx + cy * cy;
        const double gh = A.gho[q], gb = A.gbo[q];
        const double geh = beta / opb * gh, geb = beta / opb * gb;
        const double hh[4] = {C.rh[q], Tn.mh[q], Tn.kxh[q], Tn.kyh[q]}, bb[4] = {C.rb[q], Tn.mb[q], Tn.kxb[q], Tn.kyb[q]};
        double ghf[4], gbf[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const double gx = gS[2 * f], gy = gS[2 * f + 1];
            ghf[f] = 0.5 * wk * c2 * (cx * gx + cy * gy);
            gbf[f] = 0.5 * wk * (cx * gx + cy * gy);
            heat_shift_adj(wk, cx, cy, hh[f], bb[f], gx, gy, gux, gvy);
        }
        A.grh[q] = gh / opb + ghf[0];
        A.grb[q] = gb / opb + gbf[0];
        A.gTo[0][q] += geh + ghf[1];
        A.gTo[1][q] += geb + gbf[1];
        A.gTo[2][q] += r0 * geh + ghf[2];
        A.gTo[3][q] += r0 * geb + gbf[2];
        A.gTo[4][q] += r1 * geh + ghf[3];
        A.gTo[5][q] += r1 * geb + gbf[3];
    }
    acc[0] = gux;
    acc[1] = gvy;
    block_reduce_smem<2, 0>(acc, red, rout);
    if (tid == 0) {
        const double gtau = -gbeta * dt / (2.0 * tau * tau);
        const double g3[3] = {gtau, rout[0], rout[1]};
        for (int m = 0; m < 4; ++m) {
            double g = A.gWo[c * 4 + m];
#pragma unroll
            for (int o = 0; o < 3; ++o) g += g3[o] * sc[3 + o * 5 + m];
            A.gws[c * 4 + m] = g;
        }
        atomic_add(A.gpar + GP_MU, gtau * sc[3 + 4]);
    }
}

// ---------------------------------------------------------------------------------------------
// build_targets of a state, transposed: one warp per (cell, volume node).  gT: cotangents of the six
// target arrays; the node's scalars (tscal) and state (wq) come from the forward targets of that state.
// Writes gwq[(cell * 9 + node) * 4 + m].
__global__ void __launch_bounds__(256, 2) k_adj_targets(LoParams P, LoBuffers B, S2Buffers S, AdjBuffers A,
                                                         const double* gT0, const double* gT1, const double* gT2,
                                                         const double* gT3, const double* gT4, const double* gT5) {
    const int nc = P.nx * P.ny, nv = P.nvel, ck = P.ck, nr = (nv + 31) >> 5, lane = threadIdx.x & 31;
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nc * 9) return;
    const int cc = wid / 9, p = wid % 9;
    const double gw3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    const double wt2 = gw3[p % 3] * gw3[p / 3];
    const double* o = S.tscal + (size_t)wid * kS2TScal;
    double thv[4], jac[16];
    WMke M;
    w_load_scalars(o, thv, M);
#pragma unroll
    for (int m = 0; m < 16; ++m) jac[m] = o[16 + m];
    const S2Th th = s2_th(thv, ck);
    const double shb_add = 2.0 / (double)ck;
    // pass A: d/d(tdx, tdy, coeff, lam, ux, vy, theta) of the Gauss-weighted sums
    double acc[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const size_t q = (size_t)cc * nv + s.k;
        const double gmh = gT0[q], gmb = gT1[q], gkxh = gT2[q], gkxb = gT3[q], gkyh = gT4[q], gkyb = gT5[q];
        const QV v = qv_at(th, s.u, s.v);
        const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        const double shh = 2.0 * M.lam * c2 - 4.0, shb = shh + shb_add;
        double Dh[4], Db[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) { Dh[a] = v.qh * v.ld[a]; Db[a] = v.qb * v.ldb[a]; }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            acc[a] += -wt2 * (gkxh * Dh[a] + gkxb * Db[a]);
            acc[4 + a] += -wt2 * (gkyh * Dh[a] + gkyb * Db[a]);
        }
        const double xh = gkxh * v.qh, xb = gkxb * v.qb, yh = gkyh * v.qh, yb = gkyb * v.qb;
        acc[8] += wt2 * (cx * (xh * shh + xb * shb) + cy * (yh * shh + yb * shb));
        acc[9] += wt2 * M.coeff * 2.0 * c2 * (cx * (xh + xb) + cy * (yh + yb));
        acc[10] += wt2 * M.coeff * (xh * (-shh - 4.0 * M.lam * cx * cx) + xb * (-shb - 4.0 * M.lam * cx * cx) +
                                    (yh + yb) * (-4.0 * M.lam * cx * cy));
        acc[11] += wt2 * M.coeff * (yh * (-shh - 4.0 * M.lam * cy * cy) + yb * (-shb - 4.0 * M.lam * cy * cy) +
                                    (xh + xb) * (-4.0 * M.lam * cx * cy));
        const double Ah = wt2 * (gmh + M.coeff * shh * (cx * gkxh + cy * gkyh));
        const double Ab = wt2 * (gmb + M.coeff * shb * (cx * gkxb + cy * gkyb));
        double Bh[4], Bb[4], hh[4], hb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            Bh[a] = -wt2 * (gkxh * M.tdx[a] + gkyh * M.tdy[a]);
            Bb[a] = -wt2 * (gkxb * M.tdx[a] + gkyb * M.tdy[a]);
        }
        vhess(th, v, 0, Bh, hh);
        vhess(th, v, 1, Bb, hb);
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[12 + a] += Ah * Dh[a] + Ab * Db[a] + hh[a] + hb[a];
    }
    warp_sum_all<16>(acc);
    // make_mke's directions: tdx = J^-1 accx(theta, ux, vy, lam, coeff) with accx the moments of the raw
    // Shakhov terms
    double gax[4], gay[4], gJ[16];
    solve_t4(jac, acc, gax);
    solve_t4(jac, acc + 4, gay);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int a = 0; a < 4; ++a) gJ[r * 4 + a] = -(gax[r] * M.tdx[a] + gay[r] * M.tdy[a]);
    double g[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) g[m] = 0.0;   // coeff, lam, ux, vy, theta[4]
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const QV v = qv_at(th, s.u, s.v);
        const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        const double shh = 2.0 * M.lam * c2 - 4.0, shb = shh + shb_add;
        const double kxh = psi_h(s.w, s.u, s.v, gax), kxb = psi_b(s.w, gax), kyh = psi_h(s.w, s.u, s.v, gay),
                     kyb = psi_b(s.w, gay);
        const double xh = kxh * v.qh, xb = kxb * v.qb, yh = kyh * v.qh, yb = kyb * v.qb;
        g[0] += cx * (xh * shh + xb * shb) + cy * (yh * shh + yb * shb);
        g[1] += M.coeff * 2.0 * c2 * (cx * (xh + xb) + cy * (yh + yb));
        g[2] += M.coeff * (xh * (-shh - 4.0 * M.lam * cx * cx) + xb * (-shb - 4.0 * M.lam * cx * cx) +
                           (yh + yb) * (-4.0 * M.lam * cx * cy));
        g[3] += M.coeff * (yh * (-shh - 4.0 * M.lam * cy * cy) + yb * (-shb - 4.0 * M.lam * cy * cy) +
                           (xh + xb) * (-4.0 * M.lam * cx * cy));
        const double Ah = M.coeff * shh * (cx * kxh + cy * kyh), Ab = M.coeff * shb * (cx * kxb + cy * kyb);
        double Vh[4], Vb[4], hh[4], hb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            Vh[a] = s.w * (gJ[a] + s.u * gJ[4 + a] + s.v * gJ[8 + a] + 0.5 * (s.u * s.u + s.v * s.v) * gJ[12 + a]);
            Vb[a] = 0.5 * s.w * gJ[12 + a];
        }
        vhess(th, v, 0, Vh, hh);
        vhess(th, v, 1, Vb, hb);
#pragma unroll
        for (int a = 0; a < 4; ++a) g[4 + a] += Ah * v.qh * v.ld[a] + Ab * v.qb * v.ldb[a] + hh[a] + hb[a];
    }
    warp_sum_all<8>(g);
    const double gprim[4] = {acc[10] + g[2], acc[11] + g[3], acc[9] + g[1], acc[8] + g[0]};   // ux, vy, lam, coeff
    double gth[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) gth[a] = acc[12 + a] + g[4 + a];
    // the node state: theta = closure(w) (d theta = J^-1 dw) and the primitive scalars of w
    const double* w = S.wq + (size_t)wid * 4;
    double gwc[4];
    solve_t4(jac, gth, gwc);
    Dl x[4], po[4];
    seed_lane<4>(w, x);
    mke_chain(P, x, po);
    double gwp[4];
    transpose_lanes<4, 4>(po, gprim, gwp);
    if (lane < 4) A.gwq[(size_t)wid * 4 + lane] = gwc[lane] + gwp[lane];
}

// the mean-shifted volume node states of build_targets (k_s2_macro, cell part), transposed: one thread per
// (cell, component); gwq -> gW (atomically, over the cell9 stencil)
__global__ void __launch_bounds__(256) k_adj_macro_cells(LoParams P, const double* W, const double* gwq, double* gW) {
    const int nx = P.nx, ny = P.ny, nc = nx * ny;
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= nc * 4) return;
    const int cc = t >> 2, m = t & 3, i = cc % nx, j = cc / nx;
    const double gw3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    // wq[c * 3 + a] = nodes[a][c] + W - avg, avg = sum_{c,a} gw_a gw_c nodes[a][c]
    double gnode[3][3], gsum = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) gsum += gwq[((size_t)cc * 9 + c * 3 + a) * 4 + m];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) gnode[a][c] = gwq[((size_t)cc * 9 + c * 3 + a) * 4 + m] - gw3[a] * gw3[c] * gsum;
    atomic_add(gW + cc * 4 + m, gsum);
    const S2Field F{W + m, 4, nx, ny};
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : j - 2;
    // the x first layer of the 5 rows at the Gauss nodes: rows[r][a]
    double rows[5][3];
    for (int r = 0; r < 5; ++r) {
        double q[5];
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, first + r);
        S2Weno ww;
        s2_weno(q, ww);
#pragma unroll
        for (int a = 0; a < 3; ++a) rows[r][a] = s2_at_v(ww, S2_G0 + a);
    }
    double grows[5][3];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int a = 0; a < 3; ++a) grows[r][a] = 0.0;
    const int pts[3] = {S2_G0, S2_G0 + 1, S2_G0 + 2};
    const double zero3[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 3; ++a) {   // the y template of Gauss column a: vol[a][b] at the Gauss nodes b
        double a5[5], ga5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = rows[r][a];
        if (!nw) weno_points_vjp<3>(a5, pts, gnode[a], zero3, ga5);
        else
            for (int b = 0; b < 3; ++b) wall_eval_vjp(j, ny, c_s2.gnode[b], gnode[a][b], 0.0, ga5);
#pragma unroll
        for (int r = 0; r < 5; ++r) grows[r][a] = ga5[r];
    }
    for (int r = 0; r < 5; ++r) {
        double q[5], gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int s = -2; s <= 2; ++s) q[s + 2] = F.at(i + s, first + r);
        weno_points_vjp<3>(q, pts, grows[r], zero3, gq);
#pragma unroll
        for (int s = -2; s <= 2; ++s) atomic_add(gW + (size_t)((first + r) * nx + wrapx(i + s, nx)) * 4 + m, gq[s + 2]);
    }
}

// ---------------------------------------------------------------------------------------------
// the stream state and the CN right-hand side (k_cn_stream): one CTA per cell.  Writes the input
// cotangents ghi, gbi, gWi (the latter starting from gws: ws = W + res) and gTi.
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_adj_stream(LoParams P, LoBuffers B, S2Buffers T, AdjBuffers A) {
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[24];
    const int nv = P.nvel, tid = threadIdx.x, c = blockIdx.x;
    const double dt = B.dt[0];
    const double* Wo = B.W + c * 4;
    if (tid < 32) {
        const double in[5] = {Wo[0], Wo[1], Wo[2], Wo[3], P.mu_ref};
        Dl x[5], o[3];
        seed_lane<5>(in, x);
        cell_chain(P, x, x[4], o);
        if (tid < 5)
#pragma unroll
            for (int q = 0; q < 3; ++q) sc[3 + q * 5 + tid] = o[q].d;
        if (tid == 0) {
            sc[0] = o[0].v; sc[1] = o[1].v; sc[2] = o[2].v;
            // the time step is the velocity table's: TimeStep's max(U_MAX, |U| + c) is U_MAX
            Prim pr;
            const bool ok = get_primary(P.gm1, Wo, pr);
            const double sos = ok ? sqrt(0.5 * (P.gm1 + 1.0) / pr.L) : 0.0;
            if (P.fixed_dt <= 0.0 && (!ok || !(fabs(pr.U) + sos < P.umax && fabs(pr.V) + sos < P.vmax)))
                set_status(A.status, ST_ADJOINT_DT);
        }
    }
    __syncthreads();
    const double tau = sc[0], ux = sc[1], vy = sc[2], beta = dt / (2.0 * tau);
    double acc[4];
    acc[0] = acc[1] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {   // q_old = heat(W, h - M)
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double wk = s.ok ? B.w[s.kk] : 0.0, cx = B.u[s.kk] - ux, cy = B.v[s.kk] - vy, c2 = cx * cx + cy * cy;
        const double dh = B.h[q] - T.mh[q], db = B.b[q] - T.mb[q];
        acc[0] += 0.5 * wk * cx * (c2 * dh + db);
        acc[1] += 0.5 * wk * cy * (c2 * dh + db);
    }
    block_reduce_smem<2, 0>(acc, red, rout);
    const double q0 = rout[0], q1 = rout[1];
#pragma unroll
    for (int m = 0; m < 3; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const size_t q = (size_t)c * nv + s.k;
        const double grh = A.grh[q], grb = A.grb[q];
        const double dh = T.mh[q] + T.kxh[q] * q0 + T.kyh[q] * q1 - B.h[q];
        const double db = T.mb[q] + T.kxb[q] * q0 + T.kyb[q] * q1 - B.b[q];
        acc[0] += grh * dh + grb * db;
        acc[1] += beta * (grh * T.kxh[q] + grb * T.kxb[q]);
        acc[2] += beta * (grh * T.kyh[q] + grb * T.kyb[q]);
    }
    block_reduce_smem<3, 0>(acc, red, rout);
    const double gbeta = rout[0], gq0 = rout[1], gq1 = rout[2];
    double gux = 0.0, gvy = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        if (!s.ok) continue;
        const size_t q = (size_t)c * nv + s.k;
        const double wk = B.w[s.k], cx = B.u[s.k] - ux, cy = B.v[s.k] - vy, c2 = cx * cx + cy * cy;
        const double grh = A.grh[q], grb = A.grb[q];
        const double hh = 0.5 * wk * c2 * (cx * gq0 + cy * gq1), hb = 0.5 * wk * (cx * gq0 + cy * gq1);
        A.ghi[q] = grh * (1.0 - beta) + hh;
        A.gbi[q] = grb * (1.0 - beta) + hb;
        A.gTi[0][q] = beta * grh - hh;
        A.gTi[1][q] = beta * grb - hb;
        A.gTi[2][q] = beta * q0 * grh;
        A.gTi[3][q] = beta * q0 * grb;
        A.gTi[4][q] = beta * q1 * grh;
        A.gTi[5][q] = beta * q1 * grb;
        heat_shift_adj(wk, cx, cy, B.h[q] - T.mh[q], B.b[q] - T.mb[q], gq0, gq1, gux, gvy);
    }
    acc[0] = gux;
    acc[1] = gvy;
    block_reduce_smem<2, 0>(acc, red, rout);
    if (tid == 0) {
        const double gtau = -gbeta * dt / (2.0 * tau * tau);
        const double g3[3] = {gtau, rout[0], rout[1]};
        for (int m = 0; m < 4; ++m) {
            double g = A.gws[c * 4 + m];
#pragma unroll
            for (int o = 0; o < 3; ++o) g += g3[o] * sc[3 + o * 5 + m];
            A.gWi[c * 4 + m] = g;
        }
        atomic_add(A.gpar + GP_MU, gtau * sc[3 + 4]);
    }
}

// ---------------------------------------------------------------------------------------------
// ugks_node at one interior face Gauss node, transposed: flux (k_s2_face_flux) and node scalars
// (k_s2_face_nodes) together, one warp per (face, node).  Cotangents in: the face fluxes' through
// the stream rates of the two cells (grh, grb, gws), folded with the Gauss weight and face length.
// Cotangents out: the face cache at the upwind side of every velocity (grec, written; the other side's
// entry is set to zero), the macro slopes of the node (gmac) and mu_ref.
// Three CTAs per SM (168 registers with spills instead of 254 without): measured 2.5 % faster over the
// backward, the extra resident warps hiding the spills' latency.
__global__ void __launch_bounds__(128, 3) k_adj_face_nodes(LoParams P, LoBuffers B, S2Buffers S, AdjBuffers A) {
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, nr = (nv + 31) >> 5, lane = threadIdx.x & 31;
    const int nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nf * 3) return;
    const int fi = wid / 3, g = wid % 3;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    const double dt = B.dt[0];
    const double* sc = S.fscal + (size_t)wid * kS2FScal;
    if (sc[0] == 0.0) return;   // the forward node failed (its status is set)
    double thv[4], tdl[4], tdr[4], tdt[4], tdm[4], mt[5], jac[16];
    WMke M;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        thv[m] = sc[1 + m]; M.tdx[m] = sc[5 + m]; M.tdy[m] = sc[9 + m];
        tdl[m] = sc[19 + m]; tdr[m] = sc[23 + m]; tdt[m] = sc[27 + m]; tdm[m] = sc[31 + m];
    }
    M.ux = sc[13]; M.vy = sc[14]; M.lam = sc[15]; M.coeff = sc[16];
    const double q0x = sc[17], q0y = sc[18];
#pragma unroll
    for (int m = 0; m < 5; ++m) mt[m] = sc[35 + m];
#pragma unroll
    for (int m = 0; m < 16; ++m) jac[m] = sc[44 + m];
    const S2Th th = s2_th(thv, ck);
    const double shb_add = 2.0 / (double)ck;
    const double gw3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    const double ia = 1.0 / P.area, fold = (axis == 0 ? P.dy : P.dx) * gw3[g] * ia;
    double gnw[4];   // cotangent of the node's macro flux
#pragma unroll
    for (int m = 0; m < 4; ++m) gnw[m] = fold * (A.gws[cr * 4 + m] - A.gws[cl * 4 + m]);
    auto rec_at = [&](int cell, int field, int k) { return S.rec[rec_cell(cell, axis, field, g, nv) + k]; };
    // per-velocity cotangents of the node's micro flux (fhv, fbv) times vn
    auto flux_cot = [&](const WVel& s, double vn, double& ah, double& ab) {
        const double Gh = fold * (A.grh[(size_t)cr * nv + s.k] - A.grh[(size_t)cl * nv + s.k]) + psi_h(s.w, s.u, s.v, gnw);
        const double Gb = fold * (A.grb[(size_t)cr * nv + s.k] - A.grb[(size_t)cl * nv + s.k]) + psi_b(s.w, gnw);
        ah = vn * Gh;
        ab = vn * Gb;
    };
    // pass 1: the flux transposed -> Mt, q0, the directions, make_mke's scalars and theta
    double acc[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const double vn = axis == 0 ? s.u : s.v, vt = axis == 0 ? s.v : s.u;
        const bool left = vn >= 0.0;
        const int cell = left ? cl : cr;
        double ah, ab;
        flux_cot(s, vn, ah, ab);
        const QV v = qv_at(th, s.u, s.v);
        double Dh[4], Db[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) { Dh[a] = v.qh * v.ld[a]; Db[a] = v.qb * v.ldb[a]; }
        const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        const double shh = 2.0 * M.lam * c2 - 4.0, shb = shh + shb_add;
        double dx_h = 0.0, dx_b = 0.0, dy_h = 0.0, dy_b = 0.0, lr_h = 0.0, lr_b = 0.0, t_h = 0.0, t_b = 0.0, m_h = 0.0,
               m_b = 0.0;
        const double* tlr = left ? tdl : tdr;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            dx_h += Dh[a] * M.tdx[a]; dx_b += Db[a] * M.tdx[a];
            dy_h += Dh[a] * M.tdy[a]; dy_b += Db[a] * M.tdy[a];
            lr_h += Dh[a] * tlr[a]; lr_b += Db[a] * tlr[a];
            t_h += Dh[a] * tdt[a]; t_b += Db[a] * tdt[a];
            m_h += Dh[a] * tdm[a]; m_b += Db[a] * tdm[a];
        }
        const double kxh = M.coeff * cx * shh * v.qh - dx_h, kxb = M.coeff * cx * shb * v.qb - dx_b;
        const double kyh = M.coeff * cy * shh * v.qh - dy_h, kyb = M.coeff * cy * shb * v.qb - dy_b;
        const double s0h = v.qh + kxh * q0x + kyh * q0y, s0b = v.qb + kxb * q0x + kyb * q0y;
        const double sh = vn * lr_h + vt * t_h, sb = vn * lr_b + vt * t_b;
        const double f0h = rec_at(cell, 0, s.k), f0b = rec_at(cell, 1, s.k);
        const double nh = rec_at(cell, 2, s.k), th_ = rec_at(cell, 3, s.k);
        const double nb = rec_at(cell, 4, s.k), tb_ = rec_at(cell, 5, s.k);
        acc[0] += ah * s0h + ab * s0b;
        acc[1] += ah * sh + ab * sb;
        acc[2] += ah * m_h + ab * m_b;
        acc[3] += ah * f0h + ab * f0b;
        acc[4] += -(ah * (vn * nh + vt * th_) + ab * (vn * nb + vt * tb_));
        acc[5] += mt[0] * (ah * kxh + ab * kxb);
        acc[6] += mt[0] * (ah * kyh + ab * kyb);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double e = ah * Dh[a] + ab * Db[a];
            acc[7 + a] += left ? vn * e : 0.0;
            acc[11 + a] += left ? 0.0 : vn * e;
            acc[15 + a] += vt * e;
            acc[19 + a] += e;
        }
        const double qd = q0x * cx + q0y * cy, hq = ah * v.qh, bq = ab * v.qb;
        acc[23] += mt[0] * qd * (hq * shh + bq * shb);
        acc[24] += mt[0] * M.coeff * 2.0 * c2 * qd * (hq + bq);
        acc[25] += mt[0] * M.coeff * (hq * (q0x * (-shh - 4.0 * M.lam * cx * cx) + q0y * (-4.0 * M.lam * cx * cy)) +
                                     bq * (q0x * (-shb - 4.0 * M.lam * cx * cx) + q0y * (-4.0 * M.lam * cx * cy)));
        acc[26] += mt[0] * M.coeff * (hq * (q0y * (-shh - 4.0 * M.lam * cy * cy) + q0x * (-4.0 * M.lam * cx * cy)) +
                                     bq * (q0y * (-shb - 4.0 * M.lam * cy * cy) + q0x * (-4.0 * M.lam * cx * cy)));
        const double ch = mt[0] * (1.0 + M.coeff * shh * qd), cb = mt[0] * (1.0 + M.coeff * shb * qd);
        double V[4], hh[4], hb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
            V[a] = -mt[0] * (M.tdx[a] * q0x + M.tdy[a] * q0y) + mt[1] * (vn * tlr[a] + vt * tdt[a]) + mt[2] * tdm[a];
        vhess(th, v, 0, V, hh);
        vhess(th, v, 1, V, hb);
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[27 + a] += ah * (ch * Dh[a] + hh[a]) + ab * (cb * Db[a] + hb[a]);
    }
    warp_sum_all<31>(acc);
    double gmt[5], gtdl[4], gtdr[4], gtdt[4], gtdm[4], gtdx[4], gtdy[4];
#pragma unroll
    for (int m = 0; m < 5; ++m) gmt[m] = acc[m];
    const double gq0x = acc[5], gq0y = acc[6];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        gtdl[a] = mt[1] * acc[7 + a];
        gtdr[a] = mt[1] * acc[11 + a];
        gtdt[a] = mt[1] * acc[15 + a];
        gtdm[a] = mt[2] * acc[19 + a];
        gtdx[a] = -mt[0] * q0x * acc[19 + a];
        gtdy[a] = -mt[0] * q0y * acc[19 + a];
    }
    double gcoeff = acc[23], glam = acc[24], gux = acc[25], gvy = acc[26], gth[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) gth[a] = acc[27 + a];
    // the time direction: tdm = J^-1 wt, wt = -moments of the flux directions
    double gwt[4], gJ[16];
    solve_t4(jac, gtdm, gwt);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int a = 0; a < 4; ++a) gJ[r * 4 + a] = -gwt[r] * tdm[a];
    double acc3[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) acc3[m] = 0.0;
    for (int r = 0; r < nr; ++r) {   // pass 3: wt transposed -> the slope directions and theta
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const double vn = axis == 0 ? s.u : s.v, vt = axis == 0 ? s.v : s.u;
        const bool left = vn >= 0.0;
        const double* tlr = left ? tdl : tdr;
        const QV v = qv_at(th, s.u, s.v);
        const double gfh = -psi_h(s.w, s.u, s.v, gwt), gfb = -psi_b(s.w, gwt);
        double U[4], hh[4], hb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double e = gfh * v.qh * v.ld[a] + gfb * v.qb * v.ldb[a];
            acc3[a] += left ? vn * e : 0.0;
            acc3[4 + a] += left ? 0.0 : vn * e;
            acc3[8 + a] += vt * e;
            U[a] = vn * tlr[a] + vt * tdt[a];
        }
        vhess(th, v, 0, U, hh);
        vhess(th, v, 1, U, hb);
#pragma unroll
        for (int a = 0; a < 4; ++a) acc3[12 + a] += gfh * hh[a] + gfb * hb[a];
    }
    warp_sum_all<16>(acc3);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        gtdl[a] += acc3[a];
        gtdr[a] += acc3[4 + a];
        gtdt[a] += acc3[8 + a];
        gth[a] += acc3[12 + a];
    }
    // the macro slopes: tdl = J^-1 mac_l (and r, t); make_mke's directions tdx = J^-1 accx
    double gml[4], gmr[4], gmtg[4], gax[4], gay[4];
    solve_t4(jac, gtdl, gml);
    solve_t4(jac, gtdr, gmr);
    solve_t4(jac, gtdt, gmtg);
    solve_t4(jac, gtdx, gax);
    solve_t4(jac, gtdy, gay);
    if (lane == 0) {
        double* o = A.gmac + (size_t)wid * 12;
#pragma unroll
        for (int m = 0; m < 4; ++m) { o[m] = gml[m]; o[4 + m] = gmr[m]; o[8 + m] = gmtg[m]; }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int a = 0; a < 4; ++a)
            gJ[r * 4 + a] += -(gml[r] * tdl[a] + gmr[r] * tdr[a] + gmtg[r] * tdt[a] + gax[r] * M.tdx[a] + gay[r] * M.tdy[a]);
    // pass 4: accx / accy, the Jacobian and q0's analytic Maxwellian transposed
    double W0[4] = {0.0, 0.0, 0.0, 0.0};   // W0, the moments of the upwind face values (not stored)
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        const double vn = axis == 0 ? s.u : s.v;
        const bool left = vn >= 0.0;
        moment_add(s.w, s.u, s.v, rec_at(left ? cl : cr, 0, s.k), rec_at(left ? cl : cr, 1, s.k), W0);
    }
    warp_sum_all<4>(W0);
    const double nrho = W0[0], nu = W0[1] / W0[0], nvv = W0[2] / W0[0];
    const double temp = 4.0 * (W0[3] / W0[0] - 0.5 * (nu * nu + nvv * nvv)) / (double)(ck + 2);
    const double lamn = 1.0 / temp;
    double acc4[12];
#pragma unroll
    for (int m = 0; m < 12; ++m) acc4[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const double vn = axis == 0 ? s.u : s.v;
        const bool left = vn >= 0.0;
        const int cell = left ? cl : cr;
        const QV v = qv_at(th, s.u, s.v);
        const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        const double shh = 2.0 * M.lam * c2 - 4.0, shb = shh + shb_add;
        const double kxh = psi_h(s.w, s.u, s.v, gax), kxb = psi_b(s.w, gax), kyh = psi_h(s.w, s.u, s.v, gay),
                     kyb = psi_b(s.w, gay);
        const double xh = kxh * v.qh, xb = kxb * v.qb, yh = kyh * v.qh, yb = kyb * v.qb;
        acc4[0] += cx * (xh * shh + xb * shb) + cy * (yh * shh + yb * shb);
        acc4[1] += M.coeff * 2.0 * c2 * (cx * (xh + xb) + cy * (yh + yb));
        acc4[2] += M.coeff * (xh * (-shh - 4.0 * M.lam * cx * cx) + xb * (-shb - 4.0 * M.lam * cx * cx) +
                              (yh + yb) * (-4.0 * M.lam * cx * cy));
        acc4[3] += M.coeff * (yh * (-shh - 4.0 * M.lam * cy * cy) + yb * (-shb - 4.0 * M.lam * cy * cy) +
                              (xh + xb) * (-4.0 * M.lam * cx * cy));
        const double Ah = M.coeff * shh * (cx * kxh + cy * kyh), Ab = M.coeff * shb * (cx * kxb + cy * kyb);
        double Vh[4], Vb[4], hh[4], hb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            Vh[a] = s.w * (gJ[a] + s.u * gJ[4 + a] + s.v * gJ[8 + a] + 0.5 * (s.u * s.u + s.v * s.v) * gJ[12 + a]);
            Vb[a] = 0.5 * s.w * gJ[12 + a];
        }
        vhess(th, v, 0, Vh, hh);
        vhess(th, v, 1, Vb, hb);
#pragma unroll
        for (int a = 0; a < 4; ++a) acc4[4 + a] += Ah * v.qh * v.ld[a] + Ab * v.qb * v.ldb[a] + hh[a] + hb[a];
        // q0 = heat(w0, f0 - E(W0)) with (cx, cy) about make_mke's (ux, vy)
        const double du = s.u - nu, dv = s.v - nvv, cn2 = du * du + dv * dv;
        const double eah = nrho * lamn / kPi * exp(-lamn * cn2), eab = 0.5 * (double)ck * temp * eah;
        const double dh = rec_at(cell, 0, s.k) - eah, db = rec_at(cell, 1, s.k) - eab;
        heat_shift_adj(s.w, cx, cy, dh, db, gq0x, gq0y, acc4[2], acc4[3]);
        const double geah = -0.5 * s.w * c2 * (cx * gq0x + cy * gq0y), geab = -0.5 * s.w * (cx * gq0x + cy * gq0y);
        const double ge = geah + 0.5 * (double)ck * temp * geab;
        acc4[8] += ge * eah / nrho;
        acc4[9] += ge * eah * 2.0 * lamn * du;
        acc4[10] += ge * eah * 2.0 * lamn * dv;
        acc4[11] += ge * (-eah * lamn * (1.0 - lamn * cn2)) + geab * 0.5 * (double)ck * eah;
    }
    warp_sum_all<12>(acc4);
    gcoeff += acc4[0];
    glam += acc4[1];
    gux += acc4[2];
    gvy += acc4[3];
#pragma unroll
    for (int a = 0; a < 4; ++a) gth[a] += acc4[4 + a];
    // W0's scalar chain (tau -> Mt, make_mke's primitive, the analytic Maxwellian) and the closure
    const double gout[13] = {gmt[0], gmt[1], gmt[2], gmt[3], gmt[4], gux, gvy, glam, gcoeff,
                             acc4[8], acc4[9], acc4[10], acc4[11]};
    const double in[5] = {W0[0], W0[1], W0[2], W0[3], P.mu_ref};
    Dl x[5], o[13];
    seed_lane<5>(in, x);
    face_chain(P, dt, x, x[4], o);
    double gin[5], gwc[4];
    transpose_lanes<13, 5>(o, gout, gin);
    solve_t4(jac, gth, gwc);
    double gW0[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) gW0[m] = gin[m] + gwc[m];
    if (lane == 0) atomic_add(A.gpar + GP_MU, gin[4]);
    // pass 2: the face cache at the upwind side (the other side's entry of this node is zero)
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const double vn = axis == 0 ? s.u : s.v, vt = axis == 0 ? s.v : s.u;
        const bool left = vn >= 0.0;
        double ah, ab;
        flux_cot(s, vn, ah, ab);
        const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
        const double gh0 = ah * mt[3] + psi_h(s.w, s.u, s.v, gW0) + 0.5 * s.w * c2 * (cx * gq0x + cy * gq0y);
        const double gb0 = ab * mt[3] + psi_b(s.w, gW0) + 0.5 * s.w * (cx * gq0x + cy * gq0y);
        const double gv[6] = {gh0, gb0, -ah * mt[4] * vn, -ah * mt[4] * vt, -ab * mt[4] * vn, -ab * mt[4] * vt};
        double* up = A.grec + rec_cell(left ? cl : cr, axis, 0, g, nv) + s.k;
#pragma unroll
        for (int fld = 0; fld < 6; ++fld) up[(size_t)fld * 3 * nv] = gv[fld];
    }
}

// ---------------------------------------------------------------------------------------------
// the multiscale wall's scalar chain (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184), generic over
// double / Dl: inputs the wall cell's W, the wall speed and temperature, mu_ref and the tangential
// moments sw_t; outputs [rho_g, lambda, wwall[4], an[4], at[4], atime[4], Mt[5], coeff, Mxi2]
template <class T>
__device__ void micro_slope_t(int ck, const T pr[4], const T sw[4], T a[4]) {
    const double c2 = (double)(ck + 2);
    a[3] = 4.0 * (pr[3] * pr[3]) / (c2 * pr[0]) *
           (2.0 * sw[3] - 2.0 * pr[1] * sw[1] - 2.0 * pr[2] * sw[2] + sw[0] * (pr[1] * pr[1] + pr[2] * pr[2] - 0.5 * c2 / pr[3]));
    a[2] = 2.0 * pr[3] / pr[0] * (sw[2] - pr[2] * sw[0]) - pr[2] * a[3];
    a[1] = 2.0 * pr[3] / pr[0] * (sw[1] - pr[1] * sw[0]) - pr[1] * a[3];
    a[0] = sw[0] / pr[0] - pr[1] * a[1] - pr[2] * a[2] - 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + 0.5 * c2 / pr[3]) * a[3];
}
template <class T>
__device__ void wall_moments_t(int ck, const T pr[4], T Mu[7], T Mv[6], T Mxi[3]) {
    T MuL[7], MuR[7];
    const T e = 0.5 * exp(-pr[3] * (pr[1] * pr[1])) / sqrt(kPi * pr[3]);
    MuL[0] = 0.5 * erfc(-sqrt(pr[3]) * pr[1]);
    MuL[1] = pr[1] * MuL[0] + e;
    MuR[0] = 0.5 * erfc(sqrt(pr[3]) * pr[1]);
    MuR[1] = pr[1] * MuR[0] - e;
    for (int i = 2; i <= 6; ++i) {
        MuL[i] = pr[1] * MuL[i - 1] + 0.5 * (double)(i - 1) * MuL[i - 2] / pr[3];
        MuR[i] = pr[1] * MuR[i - 1] + 0.5 * (double)(i - 1) * MuR[i - 2] / pr[3];
    }
    for (int i = 0; i <= 6; ++i) Mu[i] = MuL[i] + MuR[i];
    Mv[0] = T{} + 1.0;
    Mv[1] = pr[2];
    for (int i = 2; i <= 5; ++i) Mv[i] = pr[2] * Mv[i - 1] + 0.5 * (double)(i - 1) * Mv[i - 2] / pr[3];
    Mxi[0] = T{} + 1.0;
    Mxi[1] = 0.5 * (double)ck / pr[3];
    Mxi[2] = (double)ck * ((double)ck + 2.0) / (4.0 * (pr[3] * pr[3]));
}
template <class T>
__device__ void wall_auvxi_t(const T a[4], const T Mu[7], const T Mv[6], const T Mxi[3], int al, int be, T o[4]) {
    T t[6][4];
    const int Aa[6] = {al, al + 1, al, al + 2, al, al}, Bb[6] = {be, be, be + 1, be, be + 2, be}, D[6] = {0, 0, 0, 0, 0, 2};
    for (int q = 0; q < 6; ++q) {
        t[q][0] = Mu[Aa[q]] * Mv[Bb[q]] * Mxi[D[q] / 2];
        t[q][1] = Mu[Aa[q] + 1] * Mv[Bb[q]] * Mxi[D[q] / 2];
        t[q][2] = Mu[Aa[q]] * Mv[Bb[q] + 1] * Mxi[D[q] / 2];
        t[q][3] = 0.5 * (Mu[Aa[q] + 2] * Mv[Bb[q]] * Mxi[D[q] / 2] + Mu[Aa[q]] * Mv[Bb[q] + 2] * Mxi[D[q] / 2] +
                         Mu[Aa[q]] * Mv[Bb[q]] * Mxi[(D[q] + 2) / 2]);
    }
    for (int m = 0; m < 4; ++m)
        o[m] = a[0] * t[0][m] + a[1] * t[1][m] + a[2] * t[2][m] + 0.5 * a[3] * t[3][m] + 0.5 * a[3] * t[4][m] +
               0.5 * a[3] * t[5][m];
}
template <class T>
__device__ void wall_time_coeffs_t(double dt, T tau, T mt[5]) {
    const T x = dt / tau;
    if (val(x) < 0.1) {
        T t = T{} + 1.0;
        for (int m = 0; m < 5; ++m) mt[m] = T{} + 0.0;
        for (int n = 1; n <= 24; ++n) {
            t = t * (-x) / (double)n;
            mt[3] = mt[3] - tau * t;
            if (n >= 2) { mt[0] = mt[0] + tau * t; mt[4] = mt[4] + tau * tau * (double)(n - 1) * t; }
            if (n >= 3) { mt[1] = mt[1] + tau * tau * (double)(n - 2) * t; mt[2] = mt[2] - tau * tau * t; }
        }
    } else {
        const T ex = exp(-x);
        mt[3] = tau * (1.0 - ex);
        mt[4] = -tau * dt * ex + tau * mt[3];
        mt[0] = dt - mt[3];
        mt[1] = -tau * mt[0] + mt[4];
        mt[2] = 0.5 * (dt * dt) - tau * mt[0];
    }
}
constexpr int kWallIn = 11, kWallOut = 25;
template <class T>
__device__ void wall_chain(const LoParams& P, double dt, double side, const T in[kWallIn], T out[kWallOut]) {
    const int ck = P.ck;
    const T* wcell = in;
    const T ux = in[4], tw = in[5], mu = in[6];
    const T* swt = in + 7;
    const T pp = (2.0 / (double)(ck + 2)) * (wcell[3] - 0.5 * (wcell[1] * wcell[1] + wcell[2] * wcell[2]) / wcell[0]);
    const T theta = 0.5 / (1.0 / tw);
    const T lambda = 0.5 / theta;
    const T zero = T{} + 0.0;
    const T prim_g[4] = {pp / theta, zero, -ux, lambda};
    const T wc[4] = {wcell[0], wcell[2], -wcell[1], wcell[3]};
    const T wg[4] = {prim_g[0], zero, -prim_g[0] * ux, prim_g[0] * ((double)(ck + 2) / (4.0 * lambda) + 0.5 * ux * ux)};
    const T wwall[4] = {prim_g[0], prim_g[0] * ux, zero, prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0)};
    T sw[4], an[4], at[4], atime[4], Mu[7], Mv[6], Mxi[3], m1[4], m2[4], mt[5];
    for (int m = 0; m < 4; ++m) sw[m] = (wg[m] - wc[m]) / (side * 0.5 * P.dy);
    micro_slope_t(ck, prim_g, sw, an);
    micro_slope_t(ck, prim_g, swt, at);
    wall_moments_t(ck, prim_g, Mu, Mv, Mxi);
    wall_auvxi_t(an, Mu, Mv, Mxi, 1, 0, m1);
    wall_auvxi_t(at, Mu, Mv, Mxi, 0, 1, m2);
    for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (m1[m] + m2[m]);
    micro_slope_t(ck, prim_g, sw, atime);
    const T wgg[4] = {wg[0], -wg[2], wg[1], wg[3]};
    const T tau_wall = tau_of(P, wgg, mu);
    wall_time_coeffs_t(dt, tau_wall, mt);
    out[0] = prim_g[0];
    out[1] = lambda;
    for (int m = 0; m < 4; ++m) { out[2 + m] = wwall[m]; out[6 + m] = an[m]; out[10 + m] = at[m]; out[14 + m] = atime[m]; }
    for (int m = 0; m < 5; ++m) out[18 + m] = mt[m];
    out[23] = P.pr != 1.0 ? 0.8 * (1.0 - P.pr) * lambda * lambda / prim_g[0] : zero;
    out[24] = Mxi[2];
}

// the wall node transposed: one warp per (wall face, Gauss node).  The node's forward quantities are
// recomputed here (closure of the wall state, the tangential and incident moments, the wall density);
// cotangents in: the wall face flux's (from the wall cell's stream rates) and the wall outputs' seed.
// Out: the wall cell's face cache at its wall side (written), its W, the wall speed and temperature and
// mu_ref (added).
__global__ void __launch_bounds__(256, 2) k_adj_wall_nodes(LoParams P, LoBuffers B, S2Buffers S, AdjBuffers A) {
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int nf = nx * ny + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= 2 * nx * 3) return;
    const int wf = wid / 3, g = wid % 3;
    const int top = wf >= nx ? 1 : 0, i = wf - top * nx;
    const int cc = top ? (ny - 1) * nx + i : i;
    const size_t node = (size_t)(nf + wf) * 3 + g;
    const double side = top ? 1.0 : -1.0;
    const double ux = P.wall_ux[top], theta = 0.5 / P.wall_lam[top];
    const double dt = B.dt[0];
    const double* wcell = B.W + cc * 4;
    const double pp = (2.0 / (double)(ck + 2)) * (wcell[3] - 0.5 * (wcell[1] * wcell[1] + wcell[2] * wcell[2]) / wcell[0]);
    const double lambda = 0.5 / theta;
    const double prim_g[4] = {pp / theta, 0.0, -ux, lambda};
    const double wwall[4] = {prim_g[0], prim_g[0] * ux, 0.0, prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0)};
    __shared__ double s_jac[8][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    if (!(pp > 0.0 && w_closure(P, B, wwall, C))) return;   // the forward node failed (its status is set)
    auto rec = [&](int k, int field) { return S.rec[rec_wall(nx, ny, top, i, field, g, nv) + k]; };
    double acc[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        const double hin = rec(s.k, 0), bin = rec(s.k, 1), ht = rec(s.k, 3), bt = rec(s.k, 5);
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
        acc[0] += s.w * (-ht);
        acc[1] += s.w * (-(vn * ht));
        acc[2] += s.w * (-(vt * ht));
        acc[3] += s.w * (-(0.5 * (v2 * ht + bt)));
        const double vt2 = -s.u + ux, w2 = vn * vn + vt2 * vt2;
        acc[4] += 0.5 * s.w * vn * (w2 * hin + bin);
        acc[5] += 0.5 * s.w * vt2 * (w2 * hin + bin);
        // d/d(wall speed) of the two heat-flux moments (vt2 = -u + u_w)
        acc[6] += s.w * vn * vt2 * hin;
        acc[7] += 0.5 * s.w * (w2 * hin + bin) + s.w * vt2 * vt2 * hin;
    }
    warp_sum_all<8>(acc);
    const double hlx = acc[4], hly = acc[5], dhlx_dux = acc[6], dhly_dux = acc[7];
    // the scalar chain's values and, one input per lane, its Jacobian
    const double win[kWallIn] = {wcell[0], wcell[1], wcell[2], wcell[3], ux, 1.0 / P.wall_lam[top], P.mu_ref,
                                 acc[0], acc[1], acc[2], acc[3]};
    Dl xin[kWallIn], xo[kWallOut];
#pragma unroll
    for (int q = 0; q < kWallIn; ++q) xin[q] = {win[q], q == lane ? 1.0 : 0.0};
    wall_chain(P, dt, side, xin, xo);
    double an[4], at[4], atime[4], mt[5];
#pragma unroll
    for (int m = 0; m < 4; ++m) { an[m] = xo[6 + m].v; at[m] = xo[10 + m].v; atime[m] = xo[14 + m].v; }
#pragma unroll
    for (int m = 0; m < 5; ++m) mt[m] = xo[18 + m].v;
    const double rhog = xo[0].v, lam = xo[1].v, coeff = xo[23].v, mxi2 = xo[24].v;
    const S2Th tt = s2_th(C.th, ck);
    const bool shak = P.pr != 1.0;
    const double shb_add = 2.0 / (double)ck;
    // the incident micro flux of one velocity, as the forward kernel
    auto gin = [&](const WVel& s, const QV& q, double& ginh, double& ginb) {
        const double mh = q.qh, mb = q.qb;
        double corrh = 0.0, corrb = 0.0;
        if (shak) {
            const double vn = s.v, vt = -s.u + ux, v2 = vn * vn + vt * vt;
            const double qdot = vn * hlx + vt * hly, shh = 2.0 * lam * v2 - 4.0;
            corrh = coeff * qdot * shh * mh;
            corrb = coeff * qdot * (shh + shb_add) * mb;
        }
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
        const double Han = (an[0] + an[1] * vn + an[2] * vt) * mh + 0.5 * an[3] * (v2 * mh + mb);
        const double Hat = (at[0] + at[1] * vn + at[2] * vt) * mh + 0.5 * at[3] * (v2 * mh + mb);
        const double Hti = (atime[0] + atime[1] * vn + atime[2] * vt) * mh + 0.5 * atime[3] * (v2 * mh + mb);
        const double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb + 0.5 * an[3] * (v2 * mb + mxi2 * mh);
        const double Bat = (at[0] + at[1] * vn + at[2] * vt) * mb + 0.5 * at[3] * (v2 * mb + mxi2 * mh);
        const double Bti = (atime[0] + atime[1] * vn + atime[2] * vt) * mb + 0.5 * atime[3] * (v2 * mb + mxi2 * mh);
        ginh = mt[0] * mh + mt[1] * (vn * Han + vt * Hat) + mt[2] * Hti + mt[3] * rec(s.k, 0) -
               mt[4] * (vn * rec(s.k, 2) + s.u * rec(s.k, 3)) + mt[0] * corrh;
        ginb = mt[0] * mb + mt[1] * (vn * Ban + vt * Bat) + mt[2] * Bti + mt[3] * rec(s.k, 1) -
               mt[4] * (vn * rec(s.k, 4) + s.u * rec(s.k, 5)) + mt[0] * corrb;
    };
    acc[0] = acc[1] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        const QV q = qv_at(tt, s.u, s.v);
        double gh, gb;
        gin(s, q, gh, gb);
        if (side * s.v > 0.0) acc[0] += s.w * s.v * gh;
        else acc[1] += dt * s.w * s.v * (q.qh / rhog);
    }
    warp_sum_all<2>(acc);
    const double inc = acc[0], refl = acc[1], rhow = -inc / refl;
    // cotangents of the node's micro and macro flux: the wall cell's stream rates (the bottom wall is the
    // cell's lower face, the top wall its upper face) and the wall outputs' seed
    const double gw3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    const double sgn = top ? -1.0 : 1.0, fold = sgn * P.dx * gw3[g] / P.area;
    double gnw[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) gnw[m] = fold * A.gws[cc * 4 + m];
    double gux_direct = 0.0;
    if (A.seed != nullptr) {
        const double gs = A.seed[2 * top], gq = A.seed[2 * top + 1], f = gw3[g] / (dt * nx);
        gnw[1] += -f * (gs + ux * gq);
        gnw[3] += f * gq;
        gux_direct = -f * S.nodew[node * 4 + 1] * gq;   // heat = rate_E - u_w rate_x
    }
    auto Gcot = [&](const WVel& s, double& Gh, double& Gb) {
        Gh = fold * A.grh[(size_t)cc * nv + s.k] + psi_h(s.w, s.u, s.v, gnw);
        Gb = fold * A.grb[(size_t)cc * nv + s.k] + psi_b(s.w, gnw);
    };
    // W1: the wall density's cotangent
    acc[0] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok || side * s.v > 0.0) continue;
        const QV q = qv_at(tt, s.u, s.v);
        double Gh, Gb;
        Gcot(s, Gh, Gb);
        acc[0] += dt * s.v * (q.qh / rhog * Gh + q.qb / rhog * Gb);
    }
    warp_sum_all<1>(acc);
    const double grhow = acc[0], ginc = -grhow / refl, grefl = -grhow * rhow / refl;
    // per-velocity cotangents of (ginh, ginb) and of the wall Maxwellian (wallh, wallb)
    auto cots = [&](const WVel& s, double& gh, double& gb, double& gwh, double& gwb) {
        double Gh, Gb;
        Gcot(s, Gh, Gb);
        if (side * s.v > 0.0) { gh = s.v * Gh + s.w * s.v * ginc; gb = s.v * Gb; gwh = gwb = 0.0; }
        else { gh = gb = 0.0; gwh = dt * s.v * rhow * Gh + dt * s.w * s.v * grefl; gwb = dt * s.v * rhow * Gb; }
    };
    // W2: the scalars' cotangents
    double a2[31];
#pragma unroll
    for (int m = 0; m < 31; ++m) a2[m] = 0.0;
    // [0..4] Mt, [5..8] an, [9..12] at, [13..16] atime, [17] Mxi2, [18] coeff, [19] hlx, [20] hly, [21] lambda,
    // [22] wall speed, [23..26] theta of the wall closure, [27] rho_g
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        const QV q = qv_at(tt, s.u, s.v);
        double gh, gb, gwh, gwb;
        cots(s, gh, gb, gwh, gwb);
        const double mh = q.qh, mb = q.qb;
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
        const double bh[4] = {mh, vn * mh, vt * mh, 0.5 * (v2 * mh + mb)};
        const double bb[4] = {mb, vn * mb, vt * mb, 0.5 * (v2 * mb + mxi2 * mh)};
        double Bs[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) Bs[a] = gh * bh[a] + gb * bb[a];
        const double Han = (an[0] + an[1] * vn + an[2] * vt) * mh + 0.5 * an[3] * (v2 * mh + mb);
        const double Hat = (at[0] + at[1] * vn + at[2] * vt) * mh + 0.5 * at[3] * (v2 * mh + mb);
        const double Hti = (atime[0] + atime[1] * vn + atime[2] * vt) * mh + 0.5 * atime[3] * (v2 * mh + mb);
        const double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb + 0.5 * an[3] * (v2 * mb + mxi2 * mh);
        const double Bat = (at[0] + at[1] * vn + at[2] * vt) * mb + 0.5 * at[3] * (v2 * mb + mxi2 * mh);
        const double Bti = (atime[0] + atime[1] * vn + atime[2] * vt) * mb + 0.5 * atime[3] * (v2 * mb + mxi2 * mh);
        double corrh = 0.0, corrb = 0.0, qdot = 0.0, shh = 0.0, shb = 0.0, vt2 = 0.0, w2 = 0.0;
        if (shak) {
            vt2 = -s.u + ux;
            w2 = vn * vn + vt2 * vt2;
            qdot = vn * hlx + vt2 * hly;
            shh = 2.0 * lam * w2 - 4.0;
            shb = shh + shb_add;
            corrh = coeff * qdot * shh * mh;
            corrb = coeff * qdot * shb * mb;
        }
        a2[0] += gh * (mh + corrh) + gb * (mb + corrb);
        a2[1] += gh * (vn * Han + vt * Hat) + gb * (vn * Ban + vt * Bat);
        a2[2] += gh * Hti + gb * Bti;
        a2[3] += gh * rec(s.k, 0) + gb * rec(s.k, 1);
        a2[4] += -(gh * (vn * rec(s.k, 2) + s.u * rec(s.k, 3)) + gb * (vn * rec(s.k, 4) + s.u * rec(s.k, 5)));
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            a2[5 + a] += mt[1] * vn * Bs[a];
            a2[9 + a] += mt[1] * vt * Bs[a];
            a2[13 + a] += mt[2] * Bs[a];
        }
        a2[17] += 0.5 * mh * gb * (mt[1] * (vn * an[3] + vt * at[3]) + mt[2] * atime[3]);
        if (shak) {
            const double Kc = mt[0] * (gh * shh * mh + gb * shb * mb);
            a2[18] += qdot * Kc;
            a2[19] += coeff * vn * Kc;
            a2[20] += coeff * vt2 * Kc;
            a2[21] += mt[0] * coeff * qdot * 2.0 * w2 * (gh * mh + gb * mb);
            a2[22] += mt[0] * coeff * ((gh * mh) * (hly * shh + 4.0 * lam * qdot * vt2) +
                                       (gb * mb) * (hly * shb + 4.0 * lam * qdot * vt2));
        }
        const double pa = an[0] + an[1] * vn + an[2] * vt + 0.5 * an[3] * v2;
        const double pt = at[0] + at[1] * vn + at[2] * vt + 0.5 * at[3] * v2;
        const double pi_ = atime[0] + atime[1] * vn + atime[2] * vt + 0.5 * atime[3] * v2;
        const double gmh = gh * (mt[0] + mt[1] * (vn * pa + vt * pt) + mt[2] * pi_ + (shak ? mt[0] * coeff * qdot * shh : 0.0)) +
                           gb * (0.5 * mxi2 * (mt[1] * (vn * an[3] + vt * at[3]) + mt[2] * atime[3])) + gwh / rhog;
        const double gmb = gh * (0.5 * (mt[1] * (vn * an[3] + vt * at[3]) + mt[2] * atime[3])) +
                           gb * (mt[0] + mt[1] * (vn * pa + vt * pt) + mt[2] * pi_ + (shak ? mt[0] * coeff * qdot * shb : 0.0)) +
                           gwb / rhog;
#pragma unroll
        for (int a = 0; a < 4; ++a) a2[23 + a] += gmh * q.qh * q.ld[a] + gmb * q.qb * q.ldb[a];
        a2[27] += -(gwh * mh + gwb * mb) / (rhog * rhog);
    }
    warp_sum_all<28>(a2);
    // the wall closure (theta = closure(wwall)) and the scalar chain, transposed
    double gww[4];
    solve_t4(C.jac, a2 + 23, gww);
    const double gout[kWallOut] = {a2[27], a2[21], gww[0], gww[1], gww[2], gww[3],
                                   a2[5], a2[6], a2[7], a2[8], a2[9], a2[10], a2[11], a2[12],
                                   a2[13], a2[14], a2[15], a2[16], a2[0], a2[1], a2[2], a2[3], a2[4], a2[18], a2[17]};
    double gI[kWallIn];
    transpose_lanes<kWallOut, kWallIn>(xo, gout, gI);
    if (lane == 0) {
#pragma unroll
        for (int m = 0; m < 4; ++m) atomic_add(A.gWi + cc * 4 + m, gI[m]);
        atomic_add(A.gpar + (top ? GP_UX1 : GP_UX0), gI[4] + a2[22] + gux_direct + a2[19] * dhlx_dux + a2[20] * dhly_dux);
        atomic_add(A.gpar + (top ? GP_TW1 : GP_TW0), gI[5]);
        atomic_add(A.gpar + GP_MU, gI[6]);
    }
    const double ghlx = a2[19], ghly = a2[20];
    // W3: the wall cell's face cache at the wall side
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        if (!s.ok) continue;
        double gh, gb, gwh, gwb;
        cots(s, gh, gb, gwh, gwb);
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt, vt2 = -s.u + ux, w2 = vn * vn + vt2 * vt2;
        double gv[6];
        gv[0] = mt[3] * gh + 0.5 * s.w * w2 * (vn * ghlx + vt2 * ghly);
        gv[1] = mt[3] * gb + 0.5 * s.w * (vn * ghlx + vt2 * ghly);
        gv[2] = -mt[4] * vn * gh;
        gv[3] = -mt[4] * s.u * gh - s.w * (gI[7] + vn * gI[8] + vt * gI[9] + 0.5 * v2 * gI[10]);
        gv[4] = -mt[4] * vn * gb;
        gv[5] = -mt[4] * s.u * gb - 0.5 * s.w * gI[10];
        double* o = A.grec + rec_wall(nx, ny, top, i, 0, g, nv) + s.k;
#pragma unroll
        for (int fld = 0; fld < 6; ++fld) o[(size_t)fld * 3 * nv] = gv[fld];
    }
}

// ---------------------------------------------------------------------------------------------
// the macro WENO slopes of W at the interior faces (k_s2_macro, face part), transposed: one thread
// per (face, component, side); gmac -> gW (atomically, over the side3 stencil)
__global__ void __launch_bounds__(256) k_adj_macro_faces(LoParams P, const double* W, const double* gmac, double* gW) {
    const int nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= nf * 8) return;
    const int fi = t >> 3, m = (t >> 1) & 3, right = t & 1;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int i = f % nx, j = f / nx;
    const int cell = axis == 0 ? (right ? (i + 1) % nx : i) : (right ? j + 1 : j), tangent = axis == 0 ? j : i;
    const double side = right ? -0.5 : 0.5;
    const double dnrm = axis == 0 ? P.dx : P.dy, dtg = axis == 0 ? P.dy : P.dx;
    double gdn[3], gdt[3];
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        const double* o = gmac + (size_t)(fi * 3 + g) * 12;
        gdn[g] = o[(right ? 4 : 0) + m] / dnrm;
        gdt[g] = 0.5 * o[8 + m] / dtg;
    }
    const S2Field F{W + m, 4, nx, ny};
    const int jj = axis == 0 ? tangent : cell;
    const bool nw = s2_near_wall(jj, ny);
    const int first = nw ? s2_wall_first(jj, ny) : 0;
    // the five first-layer samples (value, derivative at the side) of s2_side3_group
    double v5[5], d5[5], q5[5][5];
    for (int r = 0; r < 5; ++r) {
        double* q = q5[r];
        if (nw && axis == 1) {
#pragma unroll
            for (int tt = 0; tt < 5; ++tt) q[tt] = F.at(tangent + r - 2, first + tt);
            s2_wall_eval(q, jj, ny, side, v5[r], d5[r]);
        } else {
#pragma unroll
            for (int s = -2; s <= 2; ++s)
                q[s + 2] = nw ? F.at(cell + s, first + r)
                              : (axis == 0 ? F.at(cell + s, tangent + r - 2) : F.at(tangent + r - 2, cell + s));
            S2Weno ww;
            s2_weno(q, ww);
            s2_at(ww, side < 0.0 ? S2_XM : S2_XP, v5[r], d5[r]);
        }
    }
    double gv5[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, gd5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (nw && axis == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            wall_eval_vjp(jj, ny, c_s2.gnode[a], 0.0, gdt[a], gv5);
            wall_eval_vjp(jj, ny, c_s2.gnode[a], gdn[a], 0.0, gd5);
        }
    } else {
        const double zero3[3] = {0.0, 0.0, 0.0};
        companion3_vjp(v5, d5, zero3, gdt, gdn, gv5, gd5);
    }
    const int pt[1] = {side < 0.0 ? S2_XM : S2_XP};
    for (int r = 0; r < 5; ++r) {
        double gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (nw && axis == 1) {
            wall_eval_vjp(jj, ny, side, gv5[r], gd5[r], gq);
#pragma unroll
            for (int tt = 0; tt < 5; ++tt)
                atomic_add(gW + (size_t)((first + tt) * nx + wrapx(tangent + r - 2, nx)) * 4 + m, gq[tt]);
        } else {
            const double gvv[1] = {gv5[r]}, gdd[1] = {gd5[r]};
            weno_points_vjp<1>(q5[r], pt, gvv, gdd, gq);
#pragma unroll
            for (int s = -2; s <= 2; ++s) {
                int x, y;
                if (nw) { x = cell + s; y = first + r; }
                else if (axis == 0) { x = cell + s; y = tangent + r - 2; }
                else { x = tangent + r - 2; y = cell + s; }
                atomic_add(gW + (size_t)(y * nx + wrapx(x, nx)) * 4 + m, gq[s + 2]);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// the second layer and the positivity limiter (k_s2_recon2), transposed: CTA = 8 warps (field, part)
// over 32 velocities of one cell, as the forward kernel.  grec (this cell's face-cache entries) -> gl1 of the rows /
// columns the templates read, and the state (the limiter's cell means, the wall rows' direct samples).
// Three CTAs per SM (80 registers with spills): measured 2.3 % faster over the backward than two at 128.
__global__ void __launch_bounds__(256, 3) k_adj_recon2(LoParams P, LoBuffers B, S2Buffers S, AdjBuffers A) {
    __shared__ double s_th[8][32];
    __shared__ double s_gth[8][32];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 2, p = warp & 3;
    const int k0 = blockIdx.x * 32 + lane;
    const bool kok = k0 < nv;
    const int k = kok ? k0 : nv - 1;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : j - 2;
    const double* L1 = S.l1 + (size_t)f * 11 * nv + k;
    auto X = [&](int r, int q) { return L1[((size_t)((first + r) * nx + i) * 22 + q) * nv]; };
    const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
    // forward: the unlimited face samples and (parts 0..2) the volume Gauss row
    double face[3], dn[3], dt[3], vol[3] = {0.0, 0.0, 0.0}, a5[5], b5[5], c5[5];
    S2Weno wf;    // the face template's weights and their intermediates, for its transpose
    S2WenoX xf;
    if (p < 2) {
#pragma unroll
        for (int r = 0; r < 5; ++r) { a5[r] = X(r, 2 * p); b5[r] = X(r, 2 * p + 1); }
        if (!nw) companion3_fwd(a5, b5, face, dt, dn, wf, xf);
        else {
            double dummy;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(a5, j, ny, c_s2.gnode[a], face[a], dt[a]);
                s2_wall_eval(b5, j, ny, c_s2.gnode[a], dn[a], dummy);
            }
        }
    } else {
        const int s = p - 2;
        if (!nw) {
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                const double* y = L1 + ((size_t)(j * nx + wrapx(i + r - 2, nx)) * 22 + 7 + 2 * s) * nv;
                a5[r] = y[0];
                b5[r] = y[(size_t)nv];
            }
        } else {
#pragma unroll
            for (int r = -2; r <= 2; ++r) {
                double q[5];
#pragma unroll
                for (int t = 0; t < 5; ++t) q[t] = F.at(i + r, first + t);
                s2_wall_eval(q, j, ny, s == 0 ? -0.5 : 0.5, a5[r + 2], b5[r + 2]);
            }
        }
        companion3_fwd(a5, b5, face, dt, dn, wf, xf);
    }
    if (p < 3) {
#pragma unroll
        for (int r = 0; r < 5; ++r) c5[r] = X(r, 4 + p);
        if (!nw) {
            S2Weno ww;
            s2_weno(c5, ww);
#pragma unroll
            for (int b = 0; b < 3; ++b) vol[b] = s2_at_v(ww, S2_G0 + b);
        } else {
            double dummy;
#pragma unroll
            for (int b = 0; b < 3; ++b) s2_wall_eval(c5, j, ny, c_s2.gnode[b], vol[b], dummy);
        }
    }
    const double hm = B.h[(size_t)cc * nv + k], bm = B.b[(size_t)cc * nv + k];
    const double mf = f == 0 ? hm : bm;
    const double margin = 64.0 * kEps;
    double cand = 1.0;
    int arg = -1;   // the sample that set this warp's candidate: a (face) or 3 + a (volume)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (face[a] < 0.0) { const double x = (1.0 - margin) * mf / (mf - face[a]); if (x < cand) { cand = x; arg = a; } }
        if (p < 3 && vol[a] < 0.0) { const double x = (1.0 - margin) * mf / (mf - vol[a]); if (x < cand) { cand = x; arg = 3 + a; } }
    }
    s_th[warp][lane] = cand;
    __syncthreads();
    double tmin = s_th[0][lane];
    int wmin = 0;
#pragma unroll
    for (int w = 1; w < 8; ++w) if (s_th[w][lane] < tmin) { tmin = s_th[w][lane]; wmin = w; }
    const bool zero = (hm <= 0.0 || bm <= 0.0);
    const double theta = zero ? 0.0 : fmax(0.0, fmin(1.0, tmin));
    const double ind = 1.0 / (p < 2 ? P.dx : P.dy), itd = 1.0 / (p < 2 ? P.dy : P.dx);
    const int fv = f == 0 ? 0 : 1, fn = f == 0 ? 2 : 4, ft = f == 0 ? 3 : 5;
    // this side's cotangents: a wall side's from the wall node (every velocity), another side's from the
    // face the velocity leaves through (the face cache keeps that half only), zero for the other half
    const bool wside = (p == 2 && j == 0) || (p == 3 && j == ny - 1);
    const bool held = kok && (wside || rec_leaves(p, B.u[k], B.v[k]));
    const double* gr = A.grec + (wside ? rec_wall(nx, ny, p - 2, i, 0, 0, nv) : rec_cell(cc, p >> 1, 0, 0, nv)) + k;
    double gface[3], gdn[3], gdt[3], gvol[3] = {0.0, 0.0, 0.0}, gmf = 0.0, gth = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double gv = held ? gr[(size_t)(fv * 3 + a) * nv] : 0.0;
        const double gn = held ? gr[(size_t)(fn * 3 + a) * nv] : 0.0;
        const double gt = held ? gr[(size_t)(ft * 3 + a) * nv] : 0.0;
        gface[a] = theta * gv;
        gmf += (1.0 - theta) * gv;
        gth += (face[a] - mf) * gv + dn[a] * ind * gn + dt[a] * itd * gt;
        gdn[a] = theta * ind * gn;
        gdt[a] = theta * itd * gt;
    }
    s_gth[warp][lane] = gth;
    __syncthreads();
    // theta = min over the 8 warps' candidates when it is below 1: the argmin sample carries its cotangent
    if (!zero && tmin < 1.0 && warp == wmin && arg >= 0) {
        double gt_all = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) gt_all += s_gth[w][lane];
        const double smp = arg < 3 ? face[arg] : vol[arg - 3];
        const double den = mf - smp;
        const double dsmp = (1.0 - margin) * mf / (den * den), dmf = -(1.0 - margin) * smp / (den * den);
        if (arg < 3) gface[arg] += gt_all * dsmp;
        else gvol[arg - 3] += gt_all * dsmp;
        gmf += gt_all * dmf;
    }
    if (!kok) return;
    double* gL1 = A.gl1 + (size_t)f * 11 * nv + k;
    double* gS = (f == 0 ? A.ghi : A.gbi) + k;
    auto gX = [&](int r, int q) { return gL1 + ((size_t)((first + r) * nx + i) * 22 + q) * nv; };
    atomic_add(gS + (size_t)cc * nv, gmf);
    double ga5[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, gb5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (p < 2) {
        if (!nw) companion3_vjp(wf, xf, b5, gface, gdt, gdn, ga5, gb5);
        else
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                wall_eval_vjp(j, ny, c_s2.gnode[a], gface[a], gdt[a], ga5);
                wall_eval_vjp(j, ny, c_s2.gnode[a], gdn[a], 0.0, gb5);
            }
#pragma unroll
        for (int r = 0; r < 5; ++r) { atomic_add(gX(r, 2 * p), ga5[r]); atomic_add(gX(r, 2 * p + 1), gb5[r]); }
    } else {
        const int s = p - 2;
        companion3_vjp(wf, xf, b5, gface, gdt, gdn, ga5, gb5);
        if (!nw) {
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                double* y = gL1 + ((size_t)(j * nx + wrapx(i + r - 2, nx)) * 22 + 7 + 2 * s) * nv;
                atomic_add(y, ga5[r]);
                atomic_add(y + nv, gb5[r]);
            }
        } else {
#pragma unroll
            for (int r = -2; r <= 2; ++r) {
                double gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                wall_eval_vjp(j, ny, s == 0 ? -0.5 : 0.5, ga5[r + 2], gb5[r + 2], gq);
#pragma unroll
                for (int t = 0; t < 5; ++t) atomic_add(gS + (size_t)((first + t) * nx + wrapx(i + r, nx)) * nv, gq[t]);
            }
        }
    }
    if (p < 3 && (gvol[0] != 0.0 || gvol[1] != 0.0 || gvol[2] != 0.0)) {
        double gc5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (!nw) {
            const int pts[3] = {S2_G0, S2_G0 + 1, S2_G0 + 2};
            const double zero3[3] = {0.0, 0.0, 0.0};
            weno_points_vjp<3>(c5, pts, gvol, zero3, gc5);
        } else {
#pragma unroll
            for (int b = 0; b < 3; ++b) wall_eval_vjp(j, ny, c_s2.gnode[b], gvol[b], 0.0, gc5);
        }
#pragma unroll
        for (int r = 0; r < 5; ++r) atomic_add(gX(r, 4 + p), gc5[r]);
    }
}

// the first layer (k_s2_recon1), transposed, for one cell, field and direction at velocity k: the cell's
// gl1 entries of that direction (read once and cleared for the next step's accumulation) through the
// WENO-AO transposes into gq, the cotangents of its 5-cell stencil (x row or y column)
__device__ __forceinline__ void adj_first_layer(const LoParams& P, const LoBuffers& B, const AdjBuffers& A, int f,
                                                int dir, int cc, int k, double gq[5]) {
    const int nv = P.nvel, nx = P.nx, ny = P.ny, i = cc % nx, j = cc / nx;
    const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
    double q[5];
#pragma unroll
    for (int s = -2; s <= 2; ++s) q[s + 2] = dir == 0 ? F.at(i + s, j) : F.at(i, j + s);
    double* o = A.gl1 + ((size_t)cc * 22 + f * 11 + (dir == 0 ? 0 : 7)) * nv + k;
#pragma unroll
    for (int s = 0; s < 5; ++s) gq[s] = 0.0;
    if (dir == 0) {
        const int pts[5] = {S2_XM, S2_XP, S2_G0, S2_G0 + 1, S2_G0 + 2};
        const double gv[5] = {o[0], o[2 * (size_t)nv], o[4 * (size_t)nv], o[5 * (size_t)nv], o[6 * (size_t)nv]};
        const double gd[5] = {o[(size_t)nv], o[3 * (size_t)nv], 0.0, 0.0, 0.0};
#pragma unroll
        for (int e = 0; e < 7; ++e) o[(size_t)e * nv] = 0.0;
        weno_points_vjp<5>(q, pts, gv, gd, gq);
    } else {
        const int pts[2] = {S2_XM, S2_XP};
        const double gv[2] = {o[0], o[2 * (size_t)nv]}, gd[2] = {o[(size_t)nv], o[3 * (size_t)nv]};
#pragma unroll
        for (int e = 0; e < 4; ++e) o[(size_t)e * nv] = 0.0;
        weno_points_vjp<2>(q, pts, gv, gd, gq);
    }
}

// The first layer's transposes as gathers.  k_adj_recon1_xy: CTA = one row, 32 velocities, one field; warp
// w owns cell (w, row) and runs both of its transposes.  The x stencil cotangents go to shared memory and
// each warp sums the five that land on its own cell into the state cotangent -- a plain read-modify-write
// per (cell, velocity), nothing else writing the state cotangents meanwhile; the y stencil cotangents go to
// yq ([cell][field][5][nvel], the face-cache cotangent's storage, free once k_adj_recon2 has read it).
__global__ void __launch_bounds__(512) k_adj_recon1_xy(LoParams P, LoBuffers B, AdjBuffers A, double* yq) {
    extern __shared__ double s_gq[];   // [cell][5][32]
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, i = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + lane, j = blockIdx.y, f = blockIdx.z, cc = j * nx + i;
    double gq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (k < nv) {
        // every load of both transposes first (the stencils and the cell's gl1 entries), then the clears,
        // so the two directions' memory latencies overlap
        const bool ydir = !s2_near_wall(j, ny);
        const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
        double qx[5], qy[5], ox[7], oy[4];
#pragma unroll
        for (int s = -2; s <= 2; ++s) {
            qx[s + 2] = F.at(i + s, j);
            qy[s + 2] = ydir ? F.at(i, j + s) : 0.0;
        }
        double* o = A.gl1 + ((size_t)cc * 22 + f * 11) * nv + k;
#pragma unroll
        for (int e = 0; e < 7; ++e) ox[e] = o[(size_t)e * nv];
#pragma unroll
        for (int e = 0; e < 4; ++e) oy[e] = ydir ? o[(size_t)(7 + e) * nv] : 0.0;
#pragma unroll
        for (int e = 0; e < 11; ++e)
            if (e < 7 || ydir) o[(size_t)e * nv] = 0.0;
        {
            const int pts[5] = {S2_XM, S2_XP, S2_G0, S2_G0 + 1, S2_G0 + 2};
            const double gv[5] = {ox[0], ox[2], ox[4], ox[5], ox[6]}, gd[5] = {ox[1], ox[3], 0.0, 0.0, 0.0};
            weno_points_vjp<5>(qx, pts, gv, gd, gq);
        }
        if (ydir) {
            const int pts[2] = {S2_XM, S2_XP};
            const double gv[2] = {oy[0], oy[2]}, gd[2] = {oy[1], oy[3]};
            double gy[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            weno_points_vjp<2>(qy, pts, gv, gd, gy);
#pragma unroll
            for (int s = 0; s < 5; ++s) yq[(((size_t)cc * 2 + f) * 5 + s) * nv + k] = gy[s];
        }
    }
#pragma unroll
    for (int s = 0; s < 5; ++s) s_gq[(i * 5 + s) * 32 + lane] = gq[s];
    __syncthreads();
    if (k >= nv) return;
    double sum = 0.0;
#pragma unroll
    for (int s = -2; s <= 2; ++s) sum += s_gq[(wrapx(i - s, nx) * 5 + (s + 2)) * 32 + lane];
    double* g = (f == 0 ? A.ghi : A.gbi) + (size_t)cc * nv + k;
    *g = *g + sum;
}

// ... and the y gather: thread per (cell, velocity, field) sums the y stencil cotangents its column's owners
// (rows t-2 .. t+2 away from the walls) left in yq.  Runs after k_adj_recon1_xy.
__global__ void __launch_bounds__(256) k_adj_recon1_yg(LoParams P, AdjBuffers A, const double* yq) {
    const int nv = P.nvel, nx = P.nx, ny = P.ny;
    const int k = blockIdx.x * blockDim.x + threadIdx.x, cc = blockIdx.y, f = blockIdx.z;
    if (k >= nv) return;
    const int i = cc % nx, t = cc / nx;
    double sum = 0.0;
#pragma unroll
    for (int s = -2; s <= 2; ++s) {
        const int o = t - s;
        if (o >= 0 && o < ny && !s2_near_wall(o, ny)) sum += yq[(((size_t)(o * nx + i) * 2 + f) * 5 + (s + 2)) * nv + k];
    }
    double* g = (f == 0 ? A.ghi : A.gbi) + (size_t)cc * nv + k;
    *g = *g + sum;
}

// the scatter form of the same transposes, for grids whose row or column does not fit one CTA: CTA = 4
// warps (field, direction) over 32 velocities of one cell, only direction `only` at work; atomic adds into
// the five stencil cells
__global__ void __launch_bounds__(128) k_adj_recon1(LoParams P, LoBuffers B, AdjBuffers A, int only) {
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 1, dir = warp & 1;
    const int k0 = blockIdx.x * 32 + lane;
    if (k0 >= nv || dir != only) return;
    const int k = k0, cc = blockIdx.y, i = cc % nx, j = cc / nx;
    if (dir == 1 && s2_near_wall(j, ny)) return;
    double gq[5];
    adj_first_layer(P, B, A, f, dir, cc, k, gq);
    double* gS = (f == 0 ? A.ghi : A.gbi) + k;
#pragma unroll
    for (int s = -2; s <= 2; ++s) {
        const int x = dir == 0 ? wrapx(i + s, nx) : i, y = dir == 0 ? j : j + s;
        atomic_add(gS + (size_t)(y * nx + x) * nv, gq[s + 2]);
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// host side

size_t adj_work_doubles(int nx, int ny, int nv) {
    const size_t nc = (size_t)nx * ny, S = nc * nv, nf = nc + (size_t)nx * (ny - 1);
    auto r = [](size_t n) { return (n + 31) / 32 * 32; };
    return 2 * r(S) + r(nc * 4) + r(nc * 9 * 4) + r(s2_rec_doubles(nx, ny, nv)) + r(nc * 22 * nv) + r(nf * 3 * 12) +
           r(GP_COUNT);
}

void adj_bind_work(AdjBuffers& A, double* base, int nx, int ny, int nv) {
    const size_t nc = (size_t)nx * ny, S = nc * nv, nf = nc + (size_t)nx * (ny - 1);
    auto r = [](size_t n) { return (n + 31) / 32 * 32; };
    A.grh = base; base += r(S);
    A.grb = base; base += r(S);
    A.gws = base; base += r(nc * 4);
    A.gwq = base; base += r(nc * 9 * 4);
    A.grec = base; base += r(s2_rec_doubles(nx, ny, nv));
    A.gl1 = base; base += r(nc * 22 * nv);
    A.gmac = base; base += r(nf * 3 * 12);
    A.gpar = base;
}

cudaError_t prepare_s2_adjoint() { return s2_upload_tables(); }

template <int VPT>
static cudaError_t adj_launch(const LoParams& P, const LoBuffers& B, const S2Buffers& S, const S2Buffers& T,
                              const S2Buffers& To, const CnBuffers& C, const AdjBuffers& A, cudaStream_t s,
                              cudaStream_t s2, const cudaEvent_t* ev) {
    const int nx = P.nx, ny = P.ny, nv = P.nvel, nc = nx * ny, nf = nx * ny + nx * (ny - 1);
    auto warps = [](long long n, int nt) { return (unsigned)((n * 32 + nt - 1) / nt); };
    const bool side = s2 != nullptr && ev != nullptr;
    const cudaStream_t sw = side ? s2 : s;
    cudaError_t e = cudaSuccess;
    k_adj_collide<VPT, 256><<<nc, 256, 0, s>>>(P, B, To, C, A);
    k_adj_targets<<<warps((long long)nc * 9, 256), 256, 0, s>>>(P, B, S, A, A.gTo[0], A.gTo[1], A.gTo[2], A.gTo[3],
                                                                A.gTo[4], A.gTo[5]);
    k_adj_macro_cells<<<(unsigned)((nc * 4 + 255) / 256), 256, 0, s>>>(P, C.ws, A.gwq, A.gws);
    k_adj_stream<VPT, 256><<<nc, 256, 0, s>>>(P, B, T, A);
    // the wall nodes (2 nx x 3 warps) beside the interior face nodes: they write disjoint sides of the face
    // cache and add to gWi and the parameters atomically; the macro slopes' transpose beside recon2
    if (side) {
        e = cudaEventRecord(ev[0], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, ev[0], 0);
    }
    if (e == cudaSuccess) {
        k_adj_wall_nodes<<<warps(2LL * nx * 3, 256), 256, 0, sw>>>(P, B, S, A);
        if (side) e = cudaEventRecord(ev[1], s2);
    }
    if (e == cudaSuccess) {
        k_adj_face_nodes<<<warps((long long)nf * 3, 128), 128, 0, s>>>(P, B, S, A);
        if (side) e = cudaEventRecord(ev[2], s);
    }
    if (e == cudaSuccess && side) e = cudaStreamWaitEvent(s2, ev[2], 0);
    if (e == cudaSuccess) {
        k_adj_macro_faces<<<(unsigned)((nf * 8 + 255) / 256), 256, 0, sw>>>(P, B.W, A.gmac, A.gWi);
        if (side) e = cudaEventRecord(ev[3], s2);
    }
    if (e == cudaSuccess && side) e = cudaStreamWaitEvent(s, ev[1], 0);   // recon2 reads the wall sides
    if (e == cudaSuccess) {
        const dim3 grid((unsigned)((nv + 31) / 32), (unsigned)nc);
        k_adj_recon2<<<grid, 256, 0, s>>>(P, B, S, A);
        const unsigned kb = (unsigned)((nv + 31) / 32);
        if (nx <= 16) {   // one row per CTA
            k_adj_recon1_xy<<<dim3(kb, (unsigned)ny, 2), 32 * nx, (size_t)nx * 5 * 32 * sizeof(double), s>>>(P, B, A,
                                                                                                         A.grec);
            k_adj_recon1_yg<<<dim3((unsigned)((nv + 255) / 256), (unsigned)nc, 2), 256, 0, s>>>(P, A, A.grec);
        } else {
            k_adj_recon1<<<grid, 128, 0, s>>>(P, B, A, 0);
            k_adj_recon1<<<grid, 128, 0, s>>>(P, B, A, 1);
        }
    }
    if (e == cudaSuccess && side) e = cudaStreamWaitEvent(s, ev[3], 0);   // gWi complete before the next step
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t enqueue_s2cn2_adjoint(const LoParams& P, const LoBuffers& B, const S2Buffers& S, const S2Buffers& T,
                                  const S2Buffers& To, const CnBuffers& C, const AdjBuffers& A, cudaStream_t s,
                                  cudaStream_t s2, const cudaEvent_t* ev) {
    return P.nvel <= 1024 ? adj_launch<4>(P, B, S, T, To, C, A, s, s2, ev)
                          : adj_launch<10>(P, B, S, T, To, C, A, s, s2, ev);
}

cudaError_t enqueue_targets_adjoint(const LoParams& P, const LoBuffers& B, const S2Buffers& S, double* const gT[6],
                                    double* gW, const AdjBuffers& A, cudaStream_t s) {
    const int nc = P.nx * P.ny;
    k_adj_targets<<<(unsigned)(((long long)nc * 9 * 32 + 255) / 256), 256, 0, s>>>(P, B, S, A, gT[0], gT[1], gT[2],
                                                                                 gT[3], gT[4], gT[5]);
    k_adj_macro_cells<<<(unsigned)((nc * 4 + 255) / 256), 256, 0, s>>>(P, B.W, A.gwq, gW);
    return cudaGetLastError();
}

}  // namespace ugks
