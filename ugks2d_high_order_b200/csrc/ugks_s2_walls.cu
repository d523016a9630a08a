// ugks_s2_walls.cu -- the research S2CN2 wall variants on sm_100a (FP64).
//
// The reference keeps four switches beside its delivered multiscale wall (mod_ImportPara.f90:88-93), all
// off in its case files and single-domain only:
//   FluxWall_type = 0   : the free-streaming diffuse wall s2w1_wall_node (mod_S2D1.f90:961-995) in place
//                         of the multiscale wall node, at every wall face node (k_s2_w1_wall_nodes).
//   W1T (time centred)  : S2W1PredictMidpointWall (mod_S2NativeAdapter.f90:605-685).  An isolated half
//                         step of the accepted state -- the whole evaluation at dt/2, the transport, the
//                         CN collision at dt/2 -- predicts the state at t + dt/2; the kinetic walls are
//                         re-evaluated there at the full dt and replace the step's walls.
//   W1D (face time)     : with W1T, every interior face's leading-order flux moves to the midpoint too:
//                         f + dt (f_inst(mid) - f_lead) - dt^2/2 f_time (:660-680), f_inst the upwind
//                         transport flux of the predicted reconstruction (s2w1d_instantaneous_flux,
//                         mod_S2D1.f90:1052-1095), f_lead and f_time ugks_node's optional coefficient
//                         outputs; the macro flux is re-taken from the corrected micro flux.
//   W2R (shared)        : s2w2r_correct (mod_S2D1.f90:1152-1244).  From the leading coefficients of every
//                         face and wall, a half step of transport and BGK relaxation with the frozen
//                         tau0 = 0.1 predicts the state; the instantaneous upwind faces and the
//                         instantaneous multiscale walls (s2w2_instantaneous_node,
//                         mod_S2MultiscaleWall.f90:187-227) there correct every face, the walls included.
// Launch sequence of a variant step (enqueue_s2cn2_variant), between the step's own evaluation (which, for
// W1D and W2R, also writes the coefficient outputs into S2Buffers::coef) and k_cn_stream:
//   W1T: k_half_dt; the S2 evaluation at dt/2 into the predictor's face arrays; k_cn_stream; the targets
//        of the predicted W and k_cn_collide in predictor mode (gates only) into the predicted state; its
//        reconstruction; k_s2_w1_wall_nodes at dt into the step's wall nodes; [W1D: k_s2_face_correct over
//        the interior faces]; k_s2_combine over the wall faces.
//   W2R: k_w2r_predict; the reconstruction of the predicted state; k_w2r_walls; k_s2_face_correct over
//        every face and wall.
// A failed gate sets ST_W1T_PREDICTOR (the reference's abort 449) or ST_W2R (456), which stops the step.
#include "ugks_s2cn2.cuh"
#include "ugks_s2_math.cuh"

namespace ugks {

constexpr double kTau0 = 0.1;               // tau0, mod_S2D1.f90:32
constexpr double kWallGate = 2.0e-12;       // gate, mod_S2D1.f90:34

// s2w1_wall_node at one (wall face, Gauss node) per warp: bottom faces of row 0, then top faces of row
// ny-1, reading the wall sides of the face cache; node fluxes into the node buffers after the interior
// faces, as k_s2_wall_nodes writes them
__global__ void __launch_bounds__(256) k_s2_w1_wall_nodes(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int nf = nx * ny + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= 2 * nx * 3) return;
    const int wf = wid / 3, g = wid % 3, top = wf >= nx ? 1 : 0, i = wf - top * nx;
    const size_t node = (size_t)(nf + wf) * 3 + g;
    const double side = top ? 1.0 : -1.0, ux = P.wall_ux[top], theta = 0.5 / P.wall_lam[top];
    const double lambda = 0.5 / theta, dt = B.dt[0];
    const double* hin = SB.rec + rec_wall(nx, ny, top, i, 0, g, nv);
    const double* bin = SB.rec + rec_wall(nx, ny, top, i, 1, g, nv);
    // the continuous wall Maxwellian lambda/pi exp(-lambda((u - ux)^2 + v^2))
    auto maxw = [&](const WVel& s) {
        const double du = s.u - ux;
        return lambda / kPi * exp(-lambda * (du * du + s.v * s.v));
    };
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r = 0; r < nr; ++r) {   // incidence and reflection
        const WVel s = wvel(B, nv, r);
        if (side * s.v > 0.0) acc[0] += s.w * s.v * hin[s.k];
        else acc[1] += s.w * s.v * maxw(s);
    }
    warp_sum_all<2>(acc);
    const double inc = acc[0], refl = acc[1], rho_w = -inc / refl;
    bool ok = isfinite(refl) && fabs(refl) > DBL_MIN && isfinite(rho_w) && rho_w > 0.0;
    if (ok) {
        double* outh = SB.node + node * 2 * nv;
        double* outb = outh + nv;
        acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double fh, fb;
            if (side * s.v > 0.0) {
                fh = dt * s.v * hin[s.k];
                fb = dt * s.v * bin[s.k];
            } else {
                fh = dt * s.v * rho_w * maxw(s);
                fb = (double)P.ck * theta * fh;
            }
            moment_add(s.w, s.u, s.v, fh, fb, acc);
            if (s.ok) {
                outh[s.k] = fh;
                outb[s.k] = fb;
                ok = ok && isfinite(fh) && isfinite(fb);
            }
        }
        warp_sum_all<4>(acc);
        ok = ok && isfinite(acc[0]) && isfinite(acc[1]) && isfinite(acc[2]) && isfinite(acc[3]) &&
             fabs(acc[0]) <= kWallGate * fmax(1.0, dt * fabs(inc));
        if (lane < 4) SB.nodew[node * 4 + lane] = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : (lane == 2 ? acc[2] : acc[3]));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) set_status(B.status, ST_NONFINITE_FLUX);
}

cudaError_t launch_s2_w1_walls(const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s) {
    const long long warps = 2LL * P.nx * 3;
    k_s2_w1_wall_nodes<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(P, B, S);
    return cudaGetLastError();
}

// the predictor's time step: dt/2 of the step's dt
__global__ void k_half_dt(const double* dt, double* half) {
    if (threadIdx.x == 0) { half[0] = 0.5 * dt[0]; half[1] = 0.0; }
}

// One face per CTA: its micro flux corrected to f + dt (f_inst - f_lead) - dt^2/2 f_time, with f the
// Gauss-weighted node fluxes of the step's evaluation (T.node), f_lead / f_time the weighted coefficient
// outputs (T.coef) and f_inst the instantaneous flux of the predicted state -- the weighted upwind face
// values times the normal velocity (prec, the predicted reconstruction) on an interior face, the weighted
// instantaneous wall node fluxes (inst) on a wall; then the macro flux of the corrected micro flux.
// Written times the face length into the face arrays.  Walls (W2R) also refresh the ledger's raw wall
// flux and the wall diagnostics, and must carry no mass.  Faces: interior x, interior y, walls.
__global__ void __launch_bounds__(256) k_s2_face_correct(LoParams P, LoBuffers B, S2Buffers T, const double* prec,
                                                        const double* inst, int w2r) {
    if (halted(B)) return;
    __shared__ double red[8 * 4];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int fi = blockIdx.x;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    int axis = 0, cl = 0, cr = 0, wall = -1;
    size_t o;
    double len, *Fh, *Fb, *Fw;
    if (fi < nfx) {
        const int i = fi % nx, j = fi / nx;
        cl = fi; cr = j * nx + (i + 1) % nx;
        o = (size_t)cr; len = P.dy; Fh = B.fxh; Fb = B.fxb; Fw = B.fxw;
    } else if (fi < nf) {
        const int f = fi - nfx;
        axis = 1; cl = f; cr = f + nx;
        o = (size_t)(f + nx); len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    } else {
        wall = fi - nf;
        const int top = wall >= nx ? 1 : 0, i = wall - top * nx;
        o = top ? (size_t)ny * nx + i : (size_t)i; len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    }
    const double dt = B.dt[0];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int bad = 0;
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
        const double uk = B.u[k], vk = B.v[k], vn = axis == 0 ? uk : vk;
        double fh = 0.0, fb = 0.0, lh = 0.0, lb = 0.0, th = 0.0, tb = 0.0, ih = 0.0, ib = 0.0;
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            const size_t nd = (size_t)fi * 3 + g;
            const double* n2 = T.node + nd * 2 * nv;
            const double* cf = T.coef + nd * 4 * nv;
            fh = fh + gw[g] * n2[k];
            fb = fb + gw[g] * n2[(size_t)nv + k];
            lh = lh + gw[g] * cf[k];
            lb = lb + gw[g] * cf[(size_t)nv + k];
            th = th + gw[g] * cf[2 * (size_t)nv + k];
            tb = tb + gw[g] * cf[3 * (size_t)nv + k];
            if (wall < 0) {
                const double* rc = prec + rec_cell(vn >= 0.0 ? cl : cr, axis, 0, g, nv) + k;   // fields 3 nv apart
                ih = ih + gw[g] * vn * rc[0];
                ib = ib + gw[g] * vn * rc[(size_t)3 * nv];
            } else {
                const double* in = inst + ((size_t)wall * 3 + g) * 2 * nv;
                ih = ih + gw[g] * in[k];
                ib = ib + gw[g] * in[(size_t)nv + k];
            }
        }
        const double ch = fh + dt * (ih - lh) - 0.5 * (dt * dt) * th;
        const double cb = fb + dt * (ib - lb) - 0.5 * (dt * dt) * tb;
        Fh[o * nv + k] = ch * len;
        Fb[o * nv + k] = cb * len;
        moment_add(B.w[k], uk, vk, ch, cb, acc);
        if (!(isfinite(ch) && isfinite(cb))) bad = 1;
    }
    block_reduce_smem<4, 0>(acc, red, rout);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        bool ok = !bad && isfinite(rout[0]) && isfinite(rout[1]) && isfinite(rout[2]) && isfinite(rout[3]);
#pragma unroll
        for (int m = 0; m < 4; ++m) Fw[o * 4 + m] = rout[m] * len;
        if (wall >= 0) {
            ok = ok && fabs(rout[0]) <= kWallGate;   // the corrected wall carries no mass (diag(6), :1222-1229)
            const int top = wall >= nx ? 1 : 0;
            if (T.wall_raw != nullptr)
#pragma unroll
                for (int m = 0; m < 4; ++m) T.wall_raw[(size_t)wall * 4 + m] = rout[m];
            const double measure = dt * len;   // PublishWallDiagnostics of the corrected wall
            double rate[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) rate[m] = rout[m] * len / measure;
            double* a = B.wall_aero + (size_t)wall * 3;
            a[0] = rate[2];
            a[1] = -rate[1];
            a[2] = rate[3] - P.wall_ux[top] * rate[1];
        }
        if (!ok) set_status(B.status, w2r ? ST_W2R : ST_W1T_PREDICTOR);
    }
}

// W2R's predictor (s2w2r_correct, mod_S2D1.f90:1175-1193), one CTA per cell: the divergence of the
// leading coefficients dl = -(x0_r - x0_l)/dx - (y0_t - y0_b)/dy, ws = W + dt/2 moments(dl),
// hs = h + dt/2 (dl + (M - h)/tau0), bs alike; the gate: ws admissible and moments(hs, bs) = ws to 2e-12.
__global__ void __launch_bounds__(256) k_w2r_predict(LoParams P, LoBuffers B, S2Buffers T, LoBuffers Bm) {
    if (halted(B)) return;
    __shared__ double red[8 * 4];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int cc = blockIdx.x, i = cc % nx, j = cc / nx;
    const int fr = cc, fl = j * nx + (i + nx - 1) % nx;
    const int ft = j < ny - 1 ? nfx + cc : nf + nx + i, fb = j > 0 ? nfx + cc - nx : nf + i;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    const double dt = B.dt[0];
    auto lead = [&](int f, int part, int k) {   // Gauss-weighted leading coefficient of face f
        double s = 0.0;
#pragma unroll
        for (int g = 0; g < 3; ++g) s = s + gw[g] * T.coef[(((size_t)f * 3 + g) * 4 + part) * nv + k];
        return s;
    };
    auto dl = [&](int part, int k) {
        const double d = -(lead(fr, part, k) - lead(fl, part, k)) / P.dx;
        return d - (lead(ft, part, k) - lead(fb, part, k)) / P.dy;
    };
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < nv; k += blockDim.x) moment_add(B.w[k], B.u[k], B.v[k], dl(0, k), dl(1, k), acc);
    block_reduce_smem<4, 0>(acc, red, rout);
    double ws[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) ws[m] = B.W[cc * 4 + m] + 0.5 * dt * rout[m];
    acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
    int bad = 0;
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
        const size_t q = (size_t)cc * nv + k;
        const double h = B.h[q], b = B.b[q];
        const double hs = h + 0.5 * dt * (dl(0, k) + (T.mh[q] - h) / kTau0);
        const double bs = b + 0.5 * dt * (dl(1, k) + (T.mb[q] - b) / kTau0);
        Bm.h[q] = hs;
        Bm.b[q] = bs;
        moment_add(B.w[k], B.u[k], B.v[k], hs, bs, acc);
        if (!(isfinite(hs) && isfinite(bs))) bad = 1;
    }
    block_reduce_smem<4, 0>(acc, red, rout);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double rho, ux, vy, th;
        bool ok = !bad && s2_primitive(ws, P.ck, rho, ux, vy, th);
        double mx = 0.0, sc = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            mx = fmax(mx, fabs(rout[m] - ws[m]));
            sc = fmax(sc, fabs(ws[m]));
            Bm.W[cc * 4 + m] = ws[m];
        }
        ok = ok && mx / fmax(1.0, sc) <= kWallGate;
        if (!ok) set_status(B.status, ST_W2R);
    }
}

// s2w2_instantaneous_node, S2PhysicalGas = 1, at one (wall face, Gauss node) per warp: the discrete closure
// of the unit-density wall state (wall_equilibrium) scaled to cancel the incident mass flux of the predicted
// reconstruction's wall sides (prec); the un-integrated node fluxes into inst
__global__ void __launch_bounds__(256) k_w2r_walls(LoParams P, LoBuffers B, const double* prec, double* inst) {
    if (halted(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= 2 * nx * 3) return;
    const int wf = wid / 3, g = wid % 3, top = wf >= nx ? 1 : 0, i = wf - top * nx;
    const double side = top ? 1.0 : -1.0, ux = P.wall_ux[top], theta = 0.5 / P.wall_lam[top];
    const double* hin = prec + rec_wall(nx, ny, top, i, 0, g, nv);
    const double* bin = prec + rec_wall(nx, ny, top, i, 1, g, nv);
    const double wwall[4] = {1.0, ux, 0.0, (double)(ck + 2) * theta / 2.0 + ux * ux / 2.0};
    __shared__ double s_jac[8][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    bool ok = w_closure(P, B, wwall, C);
    const S2Th tt = s2_th(C.th, ck);
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, rho = 0.0, inc = 0.0;
    if (ok) {
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            if (side * s.v > 0.0) acc[0] += s.w * s.v * hin[s.k];
            else acc[1] += s.w * s.v * s2_q(tt, s.u, s.v).qh;
        }
        warp_sum_all<2>(acc);
        inc = acc[0];
        rho = -inc / acc[1];
        ok = isfinite(rho) && rho > 0.0;
    }
    if (ok) {
        double* outh = inst + ((size_t)wf * 3 + g) * 2 * nv;
        double* outb = outh + nv;
        acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double fh, fb;
            if (side * s.v > 0.0) {
                fh = s.v * hin[s.k];
                fb = s.v * bin[s.k];
            } else {
                const S2Q q = s2_q(tt, s.u, s.v);
                fh = s.v * rho * q.qh;
                fb = s.v * rho * q.qb;
            }
            acc[0] += s.w * fh;
            acc[1] += s.w * (s.u * fh);
            acc[2] += s.w * (s.v * fh);
            acc[3] += s.w * (0.5 * ((s.u * s.u + s.v * s.v) * fh + fb));
            if (s.ok) {
                outh[s.k] = fh;
                outb[s.k] = fb;
                ok = ok && isfinite(fh) && isfinite(fb);
            }
        }
        warp_sum_all<4>(acc);
        ok = ok && fabs(acc[0]) <= kWallGate * fmax(1.0, fabs(inc));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) set_status(B.status, ST_W2R);
}

int s2cn2_variant_kernels(const LoParams& P) {
    int n = 0;
    if (P.s2_midpoint)
        n += 1 + s2_enqueue_kernels(2) + 1 + 1 + s2_enqueue_kernels(3) + s2_enqueue_kernels(4) + 1 +
             (P.s2_face_time ? 1 : 0) + 1;
    if (P.s2_shared) n += 1 + s2_enqueue_kernels(4) + 1 + 1;
    return n;
}

cudaError_t enqueue_s2cn2_variant(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnVariant& V,
                                  cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    const int nx = P.nx, ny = P.ny, nc = nx * ny, nf = nc + nx * (ny - 1);
    const unsigned wall_ctas = (unsigned)((2LL * nx * 3 * 32 + 255) / 256);
    LoBuffers Bm = B;   // the predicted state
    Bm.h = V.h; Bm.b = V.b; Bm.W = V.W; Bm.eval = nullptr;
    cudaError_t e = cudaSuccess;
    if (P.s2_midpoint) {
        LoBuffers Bp = B;   // the accepted state at dt/2, with the predictor's face arrays
        Bp.dt = V.half; Bp.eval = nullptr; Bp.wall_aero = V.wall_aero;
        Bp.fxh = V.fxh; Bp.fxb = V.fxb; Bp.fxw = V.fxw; Bp.fyh = V.fyh; Bp.fyb = V.fyb; Bp.fyw = V.fyw;
        k_half_dt<<<1, 32, 0, s>>>(B.dt, V.half);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = s2_enqueue(2, P, Bp, V.Sp, s, s2, fork, join);
        if (e == cudaSuccess) e = enqueue_cn_stream(P, Bp, T, V.Cp, s);
        if (e == cudaSuccess) e = enqueue_cn_apply(P, Bp, Bm, V.Sp, V.Cp, s);
        if (e == cudaSuccess) e = s2_enqueue(4, P, Bm, V.Sp, s, s2, fork, join);
        S2Buffers Sw = T;   // the step's wall node buffers, the predicted state's face cache
        Sw.rec = V.Sp.rec;
        if (e == cudaSuccess) e = launch_s2_w1_walls(P, B, Sw, s);
        if (e == cudaSuccess && P.s2_face_time) {
            k_s2_face_correct<<<(unsigned)nf, 256, 0, s>>>(P, B, T, V.Sp.rec, nullptr, 0);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = launch_s2_combine(P, B, T, nf, 2 * nx, s);
    }
    if (e == cudaSuccess && P.s2_shared) {
        k_w2r_predict<<<(unsigned)nc, 256, 0, s>>>(P, B, T, Bm);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = s2_enqueue(4, P, Bm, V.Sp, s, s2, fork, join);
        if (e == cudaSuccess) { k_w2r_walls<<<wall_ctas, 256, 0, s>>>(P, B, V.Sp.rec, V.inst); e = cudaGetLastError(); }
        if (e == cudaSuccess) {
            k_s2_face_correct<<<(unsigned)(nf + 2 * nx), 256, 0, s>>>(P, B, T, V.Sp.rec, V.inst, 1);
            e = cudaGetLastError();
        }
    }
    return e;
}

}  // namespace ugks
