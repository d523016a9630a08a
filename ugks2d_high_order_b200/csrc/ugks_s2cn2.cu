// ugks_s2cn2.cu -- the explicit high-order S2CN2 step on sm_100a (FP64).
//
// One step (TimeStep; S2NativeEvolution with the volume targets kept between steps,
// mod_S2NativeAdapter.f90:469-490; ComputeResidual; S2NativeApplyUpdate, :867-940, whose
// advance_step, mod_S2D1.f90:1302-1435, runs on the stream state) is 13 launches:
//   k_lo_timestep  : dt of the accepted state.
//   S2 evolution   : reconstruction, interior faces and (side stream) walls of ugks_s2.cu, with the
//                    accepted state's targets.
//   k_cn_stream    : per cell the residual, the stream state wn = W + res, the gates of
//                    AssembleSteadyRateResiduals and S2NativePhysicalCollision (mod_Residual.f90,
//                    mod_S2NativeAdapter.f90:735-759), q_old = heat(W, h - M) and the CN right-hand
//                    side rh = hs + beta_old (M + K q_old - h), hs = h + res_h.
//   k_s2_targets   : build_targets of wn into the other target set.
//   k_cn_collide   : the 2x2 solve for the new heat flux and h_new = (rh + beta eq) / (1 + beta),
//                    written into the other state set; the cnres / mmerr gates; a last-CTA epilogue
//                    that takes the global conservation drift against the wall ledger and accepts
//                    (ledger advanced, accepted counter incremented, and the next step's dt taken from
//                    the accepted state's per-cell dt_local, so the steps of a ugks_s2cn2_steps sequence
//                    after its first launch no k_lo_timestep: 12 launches) or rejects (halt flag set:
//                    every later kernel of the launch sequence returns at entry and the accepted state
//                    stays in its set).
// The state and the targets are double-buffered: a step reads set p and writes set 1-p, so a
// rejected proposal never touches the accepted state and nothing is copied on acceptance.
#include "ugks_s2cn2.cuh"

namespace ugks {

cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s);

constexpr double kCnGate = 2.0e-12;   // gate of mod_S2D1.f90:34 and mod_S2NativeAdapter.f90:53

// heat (mod_S2D1.f90:83-97) contribution of one velocity
__device__ __forceinline__ void heat_add(double wk, double cx, double cy, double h, double b, double* q) {
    const double c2 = cx * cx + cy * cy;
    q[0] += 0.5 * wk * cx * (c2 * h + b);
    q[1] += 0.5 * wk * cy * (c2 * h + b);
}

__device__ __forceinline__ void cn_stop(const CnBuffers& C, const LoBuffers& B, unsigned bit) {
    atomicOr(C.halt, 1u);
    set_status(B.status, bit);
}

// ------------------------------------------------------------------------------------------
// the stream state and the CN right-hand side: one CTA per cell
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_cn_stream(LoParams P, LoBuffers B, S2Buffers T, CnBuffers C) {
    if (halted(B)) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[8];   // [0..3] res_w, [4] ux, [5] vy, [6] tau_old, [7] ok
    const int nv = P.nvel, tid = threadIdx.x, nx = P.nx;
    const int c = blockIdx.x, i = c % nx, j = c / nx;
    const double dt = B.dt[0], dti = 1.0 / dt;
    const size_t fl = (size_t)(j * nx + i), fr = (size_t)(j * nx + wrapx(i + 1, nx));
    const size_t gl = (size_t)(j * nx + i), gr = (size_t)((j + 1) * nx + i);
    const double* Wo = B.W + c * 4;
    if (tid == 0) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double rw = (B.fxw[fl * 4 + m] - B.fxw[fr * 4 + m] + B.fyw[gl * 4 + m] - B.fyw[gr * 4 + m]) / P.area;
            sc[m] = rw;
            C.ws[c * 4 + m] = Wo[m] + rw;
        }
        double rho, ux = 0.0, vy = 0.0, th, tau = 1.0;
        const bool ok = s2_primitive(Wo, P.ck, rho, ux, vy, th) && s2_tau(P, Wo, tau);
        sc[4] = ok ? ux : 0.0; sc[5] = ok ? vy : 0.0; sc[6] = ok ? tau : 1.0; sc[7] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const double ux = sc[4], vy = sc[5], tau = sc[6];
    const double area_inv = 1.0 / P.area;
    double h[VPT], b[VPT], hs[VPT], bs[VPT], acc[8];
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const int k = s.kk;
        const size_t q = (size_t)c * nv + k;
        const double wk = s.ok ? B.w[k] : 0.0, uk = B.u[k], vk = B.v[k];
        h[r] = B.h[q];
        b[r] = B.b[q];
        const double dh = (B.fxh[fl * nv + k] - B.fxh[fr * nv + k] + B.fyh[gl * nv + k] - B.fyh[gr * nv + k]) * area_inv;
        const double db = (B.fxb[fl * nv + k] - B.fxb[fr * nv + k] + B.fyb[gl * nv + k] - B.fyb[gr * nv + k]) * area_inv;
        hs[r] = h[r] + dh;
        bs[r] = b[r] + db;
        moment_add(wk, uk, vk, dh * dti, db * dti, acc);   // moments of the stream rate
        heat_add(wk, uk - ux, vk - vy, h[r] - T.mh[q], b[r] - T.mb[q], acc + 4);
    }
    block_reduce<6, 0>(acc, red, rout);
    if (tid == 0) {
        double rs = 1.0, err = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { rs = fmax(rs, fabs(sc[m] * dti)); err = fmax(err, fabs(acc[m] - sc[m] * dti)); }
        if (sc[7] == 0.0) cn_stop(C, B, ST_TAU);
        else if (!(err / rs <= kCnGate) || !isfinite(acc[4]) || !isfinite(acc[5])) cn_stop(C, B, ST_PROJECTION);
    }
    const double q0 = acc[4], q1 = acc[5];
    const double beta_old = dt / (2.0 * tau);
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double dh = T.mh[q] + T.kxh[q] * q0 + T.kyh[q] * q1 - h[r];
        const double db = T.mb[q] + T.kxb[q] * q0 + T.kyb[q] * q1 - b[r];
        moment_add(wk, uk, vk, dh / tau, db / tau, acc);   // S2NativePhysicalCollision moments
        if (s.ok) {
            C.rh[(size_t)c * nv + s.k] = hs[r] + beta_old * dh;
            C.rb[(size_t)c * nv + s.k] = bs[r] + beta_old * db;
        }
    }
    block_reduce_smem<4, 0>(acc, red, rout);
    if (tid == 0) {
        double ws = 1.0, mx = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { ws = fmax(ws, fabs(Wo[m])); mx = fmax(mx, fabs(rout[m])); }
        if (!(tau * mx / ws <= kCnGate)) cn_stop(C, B, ST_PROJECTION);
    }
}

// ------------------------------------------------------------------------------------------
// the CN collision of advance_step (mod_S2D1.f90:1376-1421): one CTA per cell, then the step's
// acceptance in the last CTA
template <int VPT, int NT>
__global__ void __launch_bounds__(NT) k_cn_collide(LoParams P, LoBuffers B, S2Buffers Tn, CnBuffers C, LoBuffers Bo) {
    if (halted(B)) return;
    __shared__ double red[16 * 64];
    __shared__ double rout[kRedSlots];
    __shared__ double sc[8];   // [0] beta [1] ux [2] vy [3] ok [4] max 2 beta [5..6] q_new [7] solve ok
    __shared__ unsigned s_last;
    const int nv = P.nvel, tid = threadIdx.x, c = blockIdx.x;
    const double dt = B.dt[0];
    const double* wn = C.ws + c * 4;
    if (tid == 0) {
        double tau_o = 1.0, tau_n = 1.0, rho, ux = 0.0, vy = 0.0, th;
        const bool ok = s2_tau(P, B.W + c * 4, tau_o) && s2_tau(P, wn, tau_n) && s2_primitive(wn, P.ck, rho, ux, vy, th);
        const double beta_old = dt / (2.0 * tau_o), beta = dt / (2.0 * tau_n);
        sc[0] = ok ? beta : 0.0; sc[1] = ux; sc[2] = vy; sc[3] = ok ? 1.0 : 0.0;
        sc[4] = fmax(2.0 * beta_old, 2.0 * beta);
    }
    __syncthreads();
    const double beta = sc[0], ux = sc[1], vy = sc[2];
    double rh[VPT], rb[VPT], acc[17];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double cx = uk - ux, cy = vk - vy;
        rh[r] = C.rh[q];
        rb[r] = C.rb[q];
        heat_add(wk, cx, cy, rh[r], rb[r], acc);
        heat_add(wk, cx, cy, Tn.mh[q], Tn.mb[q], acc + 2);
        heat_add(wk, cx, cy, Tn.kxh[q], Tn.kxb[q], acc + 4);   // kappa(:,1) of build_targets
        heat_add(wk, cx, cy, Tn.kyh[q], Tn.kyb[q], acc + 6);   // kappa(:,2)
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    if (tid == 0) {
        const double rhs0 = rout[0] - rout[2], rhs1 = rout[1] - rout[3];
        double a11 = -beta * rout[4], a21 = -beta * rout[5], a12 = -beta * rout[6], a22 = -beta * rout[7];
        a11 = a11 + 1.0 + beta;
        a22 = a22 + 1.0 + beta;
        const double det = a11 * a22 - a12 * a21;
        bool ok = sc[3] != 0.0 && isfinite(det) && det > 0.0;
#pragma unroll
        for (int m = 0; m < 8; ++m) ok = ok && isfinite(rout[m]);
        sc[5] = (rhs0 * a22 - a12 * rhs1) / det;
        sc[6] = (a11 * rhs1 - rhs0 * a21) / det;
        sc[7] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const double r0 = sc[5], r1 = sc[6], opb = 1.0 + beta;
    // sums: [0..1] heat(hn - M_new), [2..5] moments(hn, bn); maxima: [6..9] |rh| |rb| |hn| |bn|,
    // [10..11] CN equation residuals, [12..15] -min hn, max hn, -min bn, max bn, [16] nonfinite
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] = 0.0;
#pragma unroll
    for (int m = 6; m < 17; ++m) acc[m] = -INFINITY;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot s = slot(r, nv);
        const size_t q = (size_t)c * nv + s.kk;
        const double uk = B.u[s.kk], vk = B.v[s.kk], wk = s.ok ? B.w[s.kk] : 0.0;
        const double mh = Tn.mh[q], mb = Tn.mb[q];
        const double eqh = mh + Tn.kxh[q] * r0 + Tn.kyh[q] * r1;
        const double eqb = mb + Tn.kxb[q] * r0 + Tn.kyb[q] * r1;
        const double hn = (rh[r] + beta * eqh) / opb;
        const double bn = (rb[r] + beta * eqb) / opb;
        heat_add(wk, uk - ux, vk - vy, hn - mh, bn - mb, acc);
        moment_add(wk, uk, vk, hn, bn, acc + 2);
        if (s.ok) {
            acc[6] = fmax(acc[6], fabs(rh[r]));
            acc[7] = fmax(acc[7], fabs(rb[r]));
            acc[8] = fmax(acc[8], fabs(hn));
            acc[9] = fmax(acc[9], fabs(bn));
            acc[10] = fmax(acc[10], fabs(opb * hn - rh[r] - beta * eqh));
            acc[11] = fmax(acc[11], fabs(opb * bn - rb[r] - beta * eqb));
            acc[12] = fmax(acc[12], -hn);
            acc[13] = fmax(acc[13], hn);
            acc[14] = fmax(acc[14], -bn);
            acc[15] = fmax(acc[15], bn);
            acc[16] = fmax(acc[16], (isfinite(hn) && isfinite(bn)) ? 0.0 : 1.0);
            Bo.h[(size_t)c * nv + s.k] = hn;
            Bo.b[(size_t)c * nv + s.k] = bn;
        }
    }
    block_reduce_smem<6, 11>(acc, red, rout);
    if (tid == 0) {
        const double scale = fmax(fmax(fmax(fmax(1.0, rout[6]), rout[7]), rout[8]), rout[9]);
        double cres = fmax(rout[10], rout[11]) / scale;
        const double rh0 = rout[0], rh1 = rout[1];
        cres = fmax(cres, fmax(fabs(rh0 - r0), fabs(rh1 - r1)) /
                              fmax(fmax(1.0, fmax(fabs(rh0), fabs(rh1))), fmax(fabs(r0), fabs(r1))));
        double mx = 0.0, ws = 1.0;
        bool fin = sc[7] != 0.0 && rout[16] == 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            mx = fmax(mx, fabs(rout[2 + m] - wn[m]));
            ws = fmax(ws, fabs(wn[m]));
            fin = fin && isfinite(wn[m]) && isfinite(rout[2 + m]);
            Bo.W[c * 4 + m] = wn[m];
        }
        double* d = C.cell + (size_t)c * kCnCell;
        d[0] = sc[4];
        d[1] = isfinite(cres) ? cres : INFINITY;
        d[2] = isfinite(mx / ws) ? mx / ws : INFINITY;
        d[3] = -rout[12]; d[4] = rout[13]; d[5] = -rout[14]; d[6] = rout[15];
        d[7] = fin ? 0.0 : 1.0;
        if (!C.predict) {   // the proposal's dt_local: the next step's TimeStep when the step is accepted
            bool okd;
            const double dl = cell_dt(P, wn, okd);
            Bo.dtl[c] = okd ? dl : NAN;
        }
    }
    // last CTA: reduce the cells in a fixed order, take the conservation drift, accept or reject
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(C.counter, 1u) == (unsigned)(gridDim.x - 1)) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nc = P.nx * P.ny, nx = P.nx;
    // sums [0..3] of the proposal's W; maxima [4..15]: 2 beta, cnres, mmerr, -min h, max h, -min b,
    // max b, nonfinite, max|u|, max|v|, -min dt_local, a dt_local that failed
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
#pragma unroll
    for (int m = 4; m < 16; ++m) acc[m] = -INFINITY;
    for (int cc = tid; cc < nc; cc += blockDim.x) {
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] += __ldcg(C.ws + cc * 4 + m);
        const double* d = C.cell + (size_t)cc * kCnCell;
        acc[4] = fmax(acc[4], __ldcg(d + 0));
        acc[5] = fmax(acc[5], __ldcg(d + 1));
        acc[6] = fmax(acc[6], __ldcg(d + 2));
        acc[7] = fmax(acc[7], -__ldcg(d + 3));
        acc[8] = fmax(acc[8], __ldcg(d + 4));
        acc[9] = fmax(acc[9], -__ldcg(d + 5));
        acc[10] = fmax(acc[10], __ldcg(d + 6));
        acc[11] = fmax(acc[11], __ldcg(d + 7));
        if (!C.predict) {
            const double dl = __ldcg(Bo.dtl + cc);
            acc[14] = fmax(acc[14], -dl);
            acc[15] = fmax(acc[15], isnan(dl) ? 1.0 : 0.0);
        }
    }
    for (int k = tid; k < nv; k += blockDim.x) {
        acc[12] = fmax(acc[12], fabs(B.u[k]));
        acc[13] = fmax(acc[13], fabs(B.v[k]));
    }
    block_reduce_smem<4, 12>(acc, red, rout);
    if (tid == 0 && C.predict) {   // a predictor's advance_step: its finiteness and cnres / mmerr gates only
        if (!(rout[11] == 0.0 && rout[5] <= kCnGate && rout[6] <= kCnGate)) cn_stop(C, B, ST_W1T_PREDICTOR);
        *C.counter = 0u;
    } else if (tid == 0) {
        double* R = C.report;
        R[0] = dt;
        R[1] = rout[5]; R[2] = rout[6]; R[3] = rout[4];
        R[4] = dt * (rout[12] / P.dx + rout[13] / P.dy);
        R[5] = -rout[7]; R[6] = rout[8]; R[7] = -rout[9]; R[8] = rout[10];
        double bottom[4] = {0.0, 0.0, 0.0, 0.0}, top[4] = {0.0, 0.0, 0.0, 0.0}, drift = 0.0, bal[4];
        for (int i = 0; i < nx; ++i)
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                bottom[m] = bottom[m] + __ldcg(C.wall_raw + (size_t)i * 4 + m) / P.dy;
                top[m] = top[m] + __ldcg(C.wall_raw + ((size_t)nx + i) * 4 + m) / P.dy;
            }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double total0 = C.ledger[m];
            bal[m] = C.ledger[4 + m] + top[m] - bottom[m];
            drift = fmax(drift, fabs(rout[m] + bal[m] - total0) / fmax(1.0, fabs(total0)));
            R[10 + m] = bottom[m]; R[14 + m] = top[m]; R[18 + m] = bal[m];
        }
        // the reference's rejection hooks (S2D3_TEST_GLOBAL_REJECT, mod_S2NativeAdapter.f90:433-435,926;
        // S2E3_TEST_REJECT_STEP, mod_S2CartesianMPI.f90:254-264): the drift of the chosen step of
        // this sequence is forced above the gate
        if (C.ledger[8] > 0.0 && (double)(*C.accepted + 1u) == C.ledger[8]) drift = fmax(drift, 2.0 * kCnGate);
        R[9] = drift;
        const bool accept = rout[11] == 0.0 && rout[5] <= kCnGate && rout[6] <= kCnGate && drift <= kCnGate;
        if (accept) {
#pragma unroll
            for (int m = 0; m < 4; ++m) C.ledger[4 + m] = bal[m];
            *C.accepted = *C.accepted + 1u;
            // TimeStep of the next step from the accepted state (mod_Solve.f90:373-421), as k_lo_timestep
            // would take it at that step's start
            if (rout[15] != 0.0) set_status(B.status, ST_GETPRIMARY);
            Bo.dt[1] = Bo.dt[0];
            Bo.dt[0] = P.fixed_dt > 0.0 ? P.fixed_dt : -rout[14];
        } else {
            cn_stop(C, B, ST_STEP_REJECTED);
        }
        R[22] = accept ? 1.0 : 0.0;
        R[23] = (double)*C.accepted;
        *C.counter = 0u;
    }
}

// ------------------------------------------------------------------------------------------
// the ledger of S2NativeInitializeState (mod_S2NativeAdapter.f90:323-349): total0 = sum of W
__global__ void __launch_bounds__(256) k_cn_ledger(LoParams P, LoBuffers B, CnBuffers C) {
    __shared__ double red[8 * 64];
    __shared__ double rout[kRedSlots];
    const int nc = P.nx * P.ny;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = threadIdx.x; c < nc; c += blockDim.x)
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] += B.W[c * 4 + m];
    block_reduce_smem<4, 0>(acc, red, rout);
    if (threadIdx.x < 4) { C.ledger[threadIdx.x] = rout[threadIdx.x]; C.ledger[4 + threadIdx.x] = 0.0; }
    if (threadIdx.x == 0) { *C.halt = 0u; *C.accepted = 0u; *C.counter = 0u; }
}

template <int VPT, int NT>
static cudaError_t cn_stream_launch(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnBuffers& C,
                                    cudaStream_t s) {
    k_cn_stream<VPT, NT><<<P.nx * P.ny, NT, 0, s>>>(P, B, T, C);
    return cudaGetLastError();
}

template <int VPT, int NT>
static cudaError_t cn_apply_launch(const LoParams& P, const LoBuffers& B, const LoBuffers& Bo, const S2Buffers& To,
                                   const CnBuffers& C, cudaStream_t s) {
    LoBuffers Bw = B;   // the targets of the stream state
    Bw.W = C.ws;
    cudaError_t e = s2_enqueue(3, P, Bw, To, s, s, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    k_cn_collide<VPT, NT><<<P.nx * P.ny, NT, 0, s>>>(P, B, To, C, Bo);
    return cudaGetLastError();
}

cudaError_t enqueue_cn_stream(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnBuffers& C,
                              cudaStream_t s) {
    return P.nvel <= 1024 ? cn_stream_launch<4, 256>(P, B, T, C, s) : cn_stream_launch<10, 256>(P, B, T, C, s);
}

cudaError_t enqueue_cn_apply(const LoParams& P, const LoBuffers& B, const LoBuffers& Bo, const S2Buffers& To,
                             const CnBuffers& C, cudaStream_t s) {
    return P.nvel <= 1024 ? cn_apply_launch<4, 256>(P, B, Bo, To, C, s) : cn_apply_launch<10, 256>(P, B, Bo, To, C, s);
}

// Report (C.report) of the step: [0] dt, [1] cnres, [2] mmerr, [3] max 2 beta, [4] transport CFL,
// [5..8] min/max of h and b, [9] conservation drift, [10..13] bottom and [14..17] top wall flux / dy,
// [18..21] wall balance after the step, [22] accepted, [23] accepted steps so far.
cudaError_t enqueue_s2cn2_step(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const LoBuffers& Bo,
                               const S2Buffers& To, const CnBuffers& C, cudaStream_t s, cudaStream_t s2,
                               cudaEvent_t fork, cudaEvent_t join, long long* launches, const CnVariant* V,
                               bool timestep) {
    cudaError_t e = timestep ? launch_lo_timestep(P, B, s) : cudaSuccess;
    if (e == cudaSuccess) e = s2_enqueue(2, P, B, T, s, s2, fork, join);
    if (e == cudaSuccess && V) e = enqueue_s2cn2_variant(P, B, T, *V, s, s2, fork, join);
    if (e == cudaSuccess) e = enqueue_cn_stream(P, B, T, C, s);
    if (e == cudaSuccess) e = enqueue_cn_apply(P, B, Bo, To, C, s);
    if (launches) *launches += kCnStepKernels - (timestep ? 0 : 1) + (V ? s2cn2_variant_kernels(P) : 0);
    return e;
}

cudaError_t enqueue_s2cn2_prepare(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnBuffers& C,
                                  cudaStream_t s, long long* launches) {
    k_cn_ledger<<<1, 256, 0, s>>>(P, B, C);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = s2_enqueue(3, P, B, T, s, s, nullptr, nullptr);
    if (launches) *launches += 1 + s2_enqueue_kernels(3);
    return e;
}

}  // namespace ugks
