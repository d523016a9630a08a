// ugks_s2.cu -- the high-order "S2" evolution of HighOrderImplicit and S2CN2 on sm_100a (FP64).
//
//   k_s2_init         : S2 cold start, h, b := discrete closure Maxwellian of W (S2NativeInitializeState,
//                       mod_S2NativeAdapter.f90:192-445 with make_mke).  One warp per cell.
//   k_s2_macro        : macro WENO of W: the normal / tangential slopes of every interior face at its 3
//                       Gauss nodes (compute_flux :803-808,849-854) and the 9 mean-shifted volume node
//                       states of every cell (build_targets, mod_S2D1.f90:1246-1300).
//   k_s2_target_nodes : build_targets' closures: one warp per (cell, volume node) -> node scalars.
//   k_s2_target_sum   : the Gauss-weighted targets M, K_x, K_y per (cell, velocity) from those scalars.
//   k_s2_recon1/2     : tensor WENO-AO(5,3) reconstruction with one-sided wall quartics and the
//                       positivity limiter (mod_S2D1Reconstruction.f90, limit_cell_outputs
//                       mod_S2D1.f90:315-345): the shared first layer, then per cell the second-layer
//                       templates and the limiter; writes the face cache.
//   k_s2_face_nodes   : ugks_node (mod_S2D1.f90:421-521) at one Gauss node of one interior face per warp:
//                       closure, directions and time coefficients -> node scalars.
//   k_s2_face_flux    : the node's micro flux from those scalars, one CTA per face node.
//   k_s2_wall_nodes   : the multiscale diffuse wall node (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184)
//                       per warp.
//   k_s2_combine      : the Gauss-weighted node fluxes times the face length into the face arrays.
//
// The discrete closure (solve_q_first, mod_CorrectedWF2DClosure.f90:331-426) runs on one warp: its
// lanes stride over the velocities, every moment sum is a per-lane sum and a fixed butterfly whose
// totals every lane receives, and every lane runs the reference's accept / backtrack / stop logic on
// those identical totals.  Per-velocity closure quantities (the Maxwellian, the Shakhov directions,
// the slope directions) are recomputed from the closure's few scalars in each pass instead of being
// stored.
#include "ugks_s2_math.cuh"

namespace ugks {

// ------------------------------------------------------------------------------------------
// reconstruction + limiter in two passes into the face cache (rec_cell / rec_wall, ugks_s2.cuh; fields: h,
// b, h_n, h_t, b_n, b_t; sides: x left, x right, y bottom, y top).
//
// k_s2_recon1, the first layer (prepare_first_layer_plane, mod_S2D1Reconstruction.f90:501-578):
// per (cell, velocity, field) the 1-D WENO along x of the cell's own row -- values and derivatives
// at xi = -1/2, +1/2 and values at the 3 Gauss nodes -- and, for rows away from the walls, along y
// of the cell's own column -- values and derivatives at -1/2, +1/2.  These are the first-layer
// results the tensor templates of the 5 neighbouring cells share.  l1[cell][field*11 + q][nvel]:
// q 0..3 = x value/derivative at -1/2, +1/2; 4..6 = x Gauss values; 7..10 = y value/derivative.
// CTA: 4 warps (field, direction) over 32 velocities of one cell.
__global__ void __launch_bounds__(128) k_s2_recon1(LoParams P, LoBuffers B, S2Buffers S) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 1, dir = warp & 1;
    const int k0 = blockIdx.x * 32 + lane;
    const bool kok = k0 < nv;
    const int k = kok ? k0 : nv - 1;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    if (dir == 1 && s2_near_wall(j, ny)) return;   // walls use one-sided quartics instead
    const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
    double q[5];
    S2Weno ww;
#pragma unroll
    for (int s = -2; s <= 2; ++s) q[s + 2] = dir == 0 ? F.at(i + s, j) : F.at(i, j + s);
    const bool ok = s2_weno(q, ww);
    double* o = S.l1 + ((size_t)cc * 22 + f * 11 + (dir == 0 ? 0 : 7)) * nv + k;
    double v0, d0, v1, d1;
    s2_at(ww, S2_XM, v0, d0);
    s2_at(ww, S2_XP, v1, d1);
    if (kok) {
        o[0] = v0; o[(size_t)nv] = d0; o[2 * (size_t)nv] = v1; o[3 * (size_t)nv] = d1;
        if (dir == 0)
#pragma unroll
            for (int a = 0; a < 3; ++a) o[(size_t)(4 + a) * nv] = s2_at_v(ww, S2_G0 + a);
        if (!ok) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// k_s2_recon2, the second layer (tensor_velocity_tile, :723-792; reconstruct_wall_tile, :918-971) and
// limit_cell_outputs (mod_S2D1.f90:315-345): CTA = 8 warps (field f = warp / 4, part p = warp % 4)
// over 32 velocities of one cell.  Part p reconstructs face side p (x left, x right, y bottom, y top)
// at its 3 Gauss nodes with value, normal and tangential derivative, and parts 0..2 also the volume
// Gauss row p; the positivity factor theta is the minimum over the 8 warps (both fields, all face and
// volume samples), then each warp writes its side's limited values.
__global__ void __launch_bounds__(256, 3) k_s2_recon2(LoParams P, LoBuffers B, S2Buffers S) {
    if (eval_cached(B)) return;
    __shared__ double s_th[8][32];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = warp >> 2, p = warp & 3;
    const int k0 = blockIdx.x * 32 + lane;
    const bool kok = k0 < nv;
    const int k = kok ? k0 : nv - 1;
    const int cc = blockIdx.y, i = cc % nx, j = cc / nx;
    const bool nw = s2_near_wall(j, ny);
    const int first = nw ? s2_wall_first(j, ny) : j - 2;   // rows of the x first layer
    const double* L1 = S.l1 + (size_t)f * 11 * nv + k;
    auto X = [&](int r, int q) { return L1[((size_t)((first + r) * nx + i) * 22 + q) * nv]; };
    double face[3], dn[3], dt[3], vol[3];
    bool ok = true;
    if (p < 2) {   // x face p
        double a5[5], b5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) { a5[r] = X(r, 2 * p); b5[r] = X(r, 2 * p + 1); }
        if (!nw) ok = s2_companion3(a5, b5, face, dt, dn);
        else {
            double dummy;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                s2_wall_eval(a5, j, ny, c_s2.gnode[a], face[a], dt[a]);
                s2_wall_eval(b5, j, ny, c_s2.gnode[a], dn[a], dummy);
            }
        }
    } else {       // y face p - 2
        const int s = p - 2;
        double a5[5], b5[5];
        if (!nw) {
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                const double* y = L1 + ((size_t)(j * nx + wrapx(i + r - 2, nx)) * 22 + 7 + 2 * s) * nv;
                a5[r] = y[0];
                b5[r] = y[(size_t)nv];
            }
        } else {
            const S2Field F{(f == 0 ? B.h : B.b) + k, nv, nx, ny};
#pragma unroll
            for (int r = -2; r <= 2; ++r) {
                double q[5];
#pragma unroll
                for (int t = 0; t < 5; ++t) q[t] = F.at(i + r, first + t);
                s2_wall_eval(q, j, ny, s == 0 ? -0.5 : 0.5, a5[r + 2], b5[r + 2]);
            }
        }
        ok = s2_companion3(a5, b5, face, dt, dn);
    }
    if (p < 3) {   // volume Gauss row p
        double a5[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) a5[r] = X(r, 4 + p);
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
    // positivity factor (limit_cell_outputs): min over both fields' face and volume samples
    const double hm = B.h[(size_t)cc * nv + k], bm = B.b[(size_t)cc * nv + k];
    const double mf = f == 0 ? hm : bm;
    const double margin = 64.0 * kEps;
    double cand = 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (face[a] < 0.0) cand = fmin(cand, (1.0 - margin) * mf / (mf - face[a]));
        if (p < 3 && vol[a] < 0.0) cand = fmin(cand, (1.0 - margin) * mf / (mf - vol[a]));
    }
    s_th[warp][lane] = cand;
    __syncthreads();
    double theta = s_th[0][lane];
#pragma unroll
    for (int w = 1; w < 8; ++w) theta = fmin(theta, s_th[w][lane]);
    theta = (hm <= 0.0 || bm <= 0.0) ? 0.0 : fmax(0.0, fmin(1.0, theta));
    // the derivatives are divided by the cell sizes (limit_cell_outputs): multiplied by the reciprocals
    // here, exact when dx and dy are powers of two (the delivered meshes), within an ulp otherwise
    const double ind = 1.0 / (p < 2 ? P.dx : P.dy), itd = 1.0 / (p < 2 ? P.dy : P.dx);
    // the side this velocity leaves the cell through (the face cache's upwind half), and the wall sides
    const int fv = f == 0 ? 0 : 1, fn = f == 0 ? 2 : 4, ft = f == 0 ? 3 : 5;
    const bool store = kok && rec_leaves(p, B.u[k], B.v[k]);
    const bool wall = kok && ((p == 2 && j == 0) || (p == 3 && j == ny - 1));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double v = mf + theta * (face[a] - mf), n = theta * dn[a] * ind, t = theta * dt[a] * itd;
        if (store) {
            S.rec[rec_cell(cc, p >> 1, fv, a, nv) + k] = v;
            S.rec[rec_cell(cc, p >> 1, fn, a, nv) + k] = n;
            S.rec[rec_cell(cc, p >> 1, ft, a, nv) + k] = t;
        }
        if (wall) {
            S.rec[rec_wall(nx, ny, p - 2, i, fv, a, nv) + k] = v;
            S.rec[rec_wall(nx, ny, p - 2, i, fn, a, nv) + k] = n;
            S.rec[rec_wall(nx, ny, p - 2, i, ft, a, nv) + k] = t;
        }
        ok = ok && isfinite(v) && isfinite(n) && isfinite(t);
    }
    if (!ok && kok) set_status(B.status, ST_NONFINITE_FLUX);
}

// ------------------------------------------------------------------------------------------
// S2 cold start: one warp per cell, h, b := the discrete closure Maxwellian of W
__global__ void __launch_bounds__(256, 2) k_s2_init(LoParams P, LoBuffers B, S2Buffers SB) {
    const int nv = P.nvel, nc = P.nx * P.ny, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int cc = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (cc >= nc) return;
    __shared__ double s_jac[8][16];
    double w[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) w[m] = B.W[cc * 4 + m];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    const bool ok = w_closure(P, B, w, C) && w_make_mke(P, B, w, C, M);
    const S2Th tt = s2_th(C.th, P.ck);
    if (ok)
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const S2Q q = s2_q(tt, s.u, s.v);
            if (s.ok) { B.h[(size_t)cc * nv + s.k] = q.qh; B.b[(size_t)cc * nv + s.k] = q.qb; }
        }
    if (!ok && lane == 0) set_status(B.status, ST_PROJECTION);
}

// macro WENO of W: per interior face and component the normal slopes of both sides and the
// tangential slope at the 3 Gauss nodes (s2d1_face3, compute_flux :803-808,849-854), and per cell
// and component the 3x3 Gauss values and the mean-shifted volume node states (build_targets
// :1270-1279).  Faces: 2 warps per face, an 8-lane group per (component, side); cells: one warp per
// cell, an 8-lane group per component.
__global__ void __launch_bounds__(128) k_s2_macro(LoParams P, LoBuffers B, S2Buffers SB, int faces, int cells) {
    if (eval_cached(B)) return;
    const int nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1), nc = nx * ny;
    int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31, grp = lane >> 3, gl = lane & 7;
    const int nfw = faces ? nf * 2 : 0;
    if (wid < nfw) {
        const int fi = wid >> 1, m = (wid & 1) * 2 + (grp >> 1), right = grp & 1;
        const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
        const int i = f % nx, j = f / nx;
        const S2Field F{B.W + m, 4, nx, ny};
        double dn[3] = {0.0, 0.0, 0.0}, dt[3] = {0.0, 0.0, 0.0};
        bool ok;
        if (axis == 0) ok = s2_side3_group(F, 0, right ? (i + 1) % nx : i, j, right ? -0.5 : 0.5, gl, dn, dt);
        else ok = s2_side3_group(F, 1, right ? j + 1 : j, i, right ? -0.5 : 0.5, gl, dn, dt);
        // the right side's tangential derivatives to the left side's lane 0
        double tr[3];
#pragma unroll
        for (int g = 0; g < 3; ++g) tr[g] = __shfl_down_sync(0xffffffffu, dt[g], 8);
        if (gl == 0) {
            if (!ok) set_status(B.status, ST_NONFINITE_FLUX);
            const double dnrm = axis == 0 ? P.dx : P.dy, dtg = axis == 0 ? P.dy : P.dx;
#pragma unroll
            for (int g = 0; g < 3; ++g) {
                double* o = SB.mac + (size_t)(fi * 3 + g) * 12;
                o[(right ? 4 : 0) + m] = dn[g] / dnrm;
                if (!right) o[8 + m] = 0.5 * (dt[g] + tr[g]) / dtg;
            }
        }
        return;
    }
    wid -= nfw;
    if (!cells || wid >= nc) return;
    const int cc = wid, m = grp, i = cc % nx, j = cc / nx;
    const S2Field F{B.W + m, 4, nx, ny};
    double vol[3] = {0.0, 0.0, 0.0};
    const bool ok = s2_cell9_group(F, i, j, gl, vol);
    if (__any_sync(0xffffffffu, !ok) && lane == 0) set_status(B.status, ST_PROJECTION);
    // nodes[a][c] = vol of lane a, entry c; the mean over the 9 nodes in the reference's order
    const int base = lane & ~7;
    double nodes[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) nodes[a][c] = __shfl_sync(0xffffffffu, vol[c], base + a);
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double avg = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) avg = avg + gw[a] * gw[c] * nodes[a][c];
    const double wc = B.W[cc * 4 + m];
    if (gl < 3)
        for (int c = 0; c < 3; ++c) SB.wq[((size_t)cc * 9 + c * 3 + gl) * 4 + m] = nodes[gl][c] + wc - avg;
}

// The face-node closure kernel comes in two CTA shapes.  A single instance runs it in 128-thread
// CTAs, three per SM: up to 170 registers a thread (no spills) at 12 warps per SM, faster per step
// than two 256-thread CTAs per SM capped at 128 registers (which spill the closure's state).  Many
// instances on concurrent streams (S2Buffers::concurrent) gain more from the 16 resident warps of
// the 256-thread shape, which they keep.  The volume-node kernel is fastest in the 256-thread shape
// in both cases.
constexpr int kS2NodeThreads = 128;

// build_targets, closure part: one warp per (cell, volume node) -> the node scalars
__global__ void __launch_bounds__(256, 2) k_s2_target_nodes(LoParams P, LoBuffers B, S2Buffers SB, int qrec) {
    if (eval_cached(B)) return;
    extern __shared__ double s_qrec[];
    const int nc = P.nx * P.ny, lane = threadIdx.x & 31;
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nc * 9) return;
    __shared__ double s_jac[8][16];
    double w[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) w[m] = SB.wq[(size_t)wid * 4 + m];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    const WQRec qr{qrec ? s_qrec + (threadIdx.x >> 5) * (((P.nvel + 31) >> 5) * 32) : nullptr};
    const bool ok = w_closure(P, B, w, C, qr) && w_make_mke(P, B, w, C, M, qr);
    if (lane == 0) {
        if (ok) w_store_scalars(SB.tscal + (size_t)wid * kS2TScal, C, M);
        else set_status(B.status, ST_PROJECTION);
    }
}

// build_targets, sum part: per (cell, velocity) the Gauss-weighted M, K_x, K_y of the 9 nodes
__global__ void __launch_bounds__(256) k_s2_target_sum(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, cc = blockIdx.y;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= nv) return;
    const double uk = B.u[k], vk = B.v[k];
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    double amh = 0.0, amb = 0.0, akxh = 0.0, akxb = 0.0, akyh = 0.0, akyb = 0.0;
    for (int p = 0; p < 9; ++p) {
        double th[4];
        WMke M;
        w_load_scalars(SB.tscal + ((size_t)cc * 9 + p) * kS2TScal, th, M);
        S2Q q;
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_at(s2_th(th, P.ck), M, P.ck, uk, vk, q, mh, mb, kxh, kxb, kyh, kyb);
        const double wt2 = gw[p % 3] * gw[p / 3];
        amh = amh + wt2 * mh; amb = amb + wt2 * mb;
        akxh = akxh + wt2 * kxh; akxb = akxb + wt2 * kxb;
        akyh = akyh + wt2 * kyh; akyb = akyb + wt2 * kyb;
    }
    const size_t q = (size_t)cc * nv + k;
    SB.mh[q] = amh; SB.mb[q] = amb; SB.kxh[q] = akxh; SB.kxb[q] = akxb; SB.kyh[q] = akyh; SB.kyb[q] = akyb;
}

// ------------------------------------------------------------------------------------------
// interior face nodes (ugks_node, mod_S2D1.f90:421-521), scalar part: one warp per (face, Gauss
// node) -- the right x face of every cell, then the top y face of every cell below the last row --
// computes W0, the closure, make_mke, q0, the slope and time directions and Mt, and stores them as
// the node's scalars (SB.fscal) for k_s2_face_flux.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_s2_face_nodes(LoParams P, LoBuffers B, S2Buffers SB, int qrec) {
    if (eval_cached(B)) return;
    extern __shared__ double s_qrec[];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck, lane = threadIdx.x & 31, nr = (nv + 31) >> 5;
    const int nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (wid >= nf * 3) return;
    const int fi = wid / 3, g = wid % 3;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    const double dt = B.dt[0];
    const double* mac = SB.mac + (size_t)wid * 12;   // [nl | nr | t][component] of this node
    auto upwind = [&](const WVel& s, int field) {
        const double vn = axis == 0 ? s.u : s.v;
        const bool left = vn >= 0.0;
        return SB.rec[rec_cell(left ? cl : cr, axis, field, g, nv) + s.k];
    };
    // W0: moments of the upwind face values
    double acc[16];
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[m] = 0.0;
    for (int r = 0; r < nr; ++r) {
        const WVel s = wvel(B, nv, r);
        moment_add(s.w, s.u, s.v, upwind(s, 0), upwind(s, 1), acc);
    }
    warp_sum_all<4>(acc);
    const double w0[4] = {acc[0], acc[1], acc[2], acc[3]};
    __shared__ double s_jac[NT / 32][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    WMke M;
    const WQRec qr{qrec ? s_qrec + (threadIdx.x >> 5) * (nr * 32) : nullptr};
    bool ok = w_closure(P, B, w0, C, qr) && w_make_mke(P, B, w0, C, M, qr);
    double q0x = 0.0, q0y = 0.0, tdl[4], tdr[4], tdt[4], tdm[4], wt[4], mt[5], tau = 0.0;
    if (ok) {   // q0 = heat(w0, f0 - analytic Maxwellian of w0)
        const double nrho = w0[0], nu = w0[1] / w0[0], nvv = w0[2] / w0[0];
        const double temp = 4.0 * (w0[3] / w0[0] - 0.5 * (nu * nu + nvv * nvv)) / (double)(ck + 2);
        const double lamn = 1.0 / temp;
        // directions of the macro normal slopes (left, right) and the tangential slope
        const bool okd = s2_solve4(C.jac, mac, tdl) & s2_solve4(C.jac, mac + 4, tdr) & s2_solve4(C.jac, mac + 8, tdt);
        if (!okd)
#pragma unroll
            for (int m = 0; m < 4; ++m) tdl[m] = tdr[m] = tdt[m] = NAN;
        // one pass over the velocities for q0 (qacc) and the direction moments (acc): two independent
        // chains per velocity, each summed in velocity order and reduced on its own
        double qacc[2] = {0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 16; ++m) acc[m] = 0.0;
        const S2Th tt = s2_th(C.th, ck);
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            {
                const double du = s.u - nu, dv = s.v - nvv;
                const double eah = nrho * lamn / kPi * exp(-lamn * (du * du + dv * dv));
                const double eab = 0.5 * (double)ck * temp * eah;
                const double cx = s.u - M.ux, cy = s.v - M.vy, c2 = cx * cx + cy * cy;
                const double dh = upwind(s, 0) - eah, db = upwind(s, 1) - eab;
                qacc[0] += 0.5 * s.w * cx * (c2 * dh + db);
                qacc[1] += 0.5 * s.w * cy * (c2 * dh + db);
            }
            const S2Q q = qr.at(tt, s, r);
            double dlh, dlb, drh, drb, dth, dtb;
            s2_dq(q, tdl, dlh, dlb);
            s2_dq(q, tdr, drh, drb);
            s2_dq(q, tdt, dth, dtb);
            moment_add(s.w, s.u, s.v, dlh, dlb, acc);
            moment_add(s.w, s.u, s.v, drh, drb, acc + 4);
            moment_add(s.w, s.u, s.v, dth, dtb, acc + 8);
            const double vn = axis == 0 ? s.u : s.v, vt = axis == 0 ? s.v : s.u;
            const double fh = vn * (vn >= 0.0 ? dlh : drh) + vt * dth;
            const double fb = vn * (vn >= 0.0 ? dlb : drb) + vt * dtb;
            moment_add(s.w, s.u, s.v, fh, fb, acc + 12);
        }
        warp_sum_all<2>(qacc);
        q0x = qacc[0];
        q0y = qacc[1];
        warp_sum_all<16>(acc);
        for (int d = 0; d < 3; ++d) {   // gates of the three directions
            double mx = 0.0, sc = 1.0;
            for (int m = 0; m < 4; ++m) {
                mx = fmax(mx, fabs(acc[4 * d + m] - mac[4 * d + m]));
                sc = fmax(sc, fabs(mac[4 * d + m]));
            }
            ok = ok && mx / sc <= 2.0e-12;
        }
        // the time direction and the time coefficients Mt (mod_Evolution.f90:346-350)
#pragma unroll
        for (int m = 0; m < 4; ++m) wt[m] = -acc[12 + m];
        ok = ok && s2_solve4(C.jac, wt, tdm);
        ok = ok && s2_tau(P, w0, tau);
        const double ex = exp(-dt / tau);
        mt[3] = tau * (1.0 - ex);
        mt[4] = -tau * dt * ex + tau * mt[3];
        mt[0] = dt - mt[3];
        mt[1] = -tau * mt[0] + mt[4];
        mt[2] = 0.5 * dt * dt - tau * mt[0];
    }
    // the node scalars of the flux pass (k_s2_face_flux)
    if (lane == 0) {
        double* o = SB.fscal + (size_t)wid * kS2FScal;
        o[0] = ok ? 1.0 : 0.0;
        if (ok) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                o[1 + m] = C.th[m]; o[5 + m] = M.tdx[m]; o[9 + m] = M.tdy[m];
                o[19 + m] = tdl[m]; o[23 + m] = tdr[m]; o[27 + m] = tdt[m]; o[31 + m] = tdm[m]; o[40 + m] = wt[m];
            }
            o[13] = M.ux; o[14] = M.vy; o[15] = M.lam; o[16] = M.coeff; o[17] = q0x; o[18] = q0y;
#pragma unroll
            for (int m = 0; m < 5; ++m) o[35 + m] = mt[m];
#pragma unroll
            for (int m = 0; m < 16; ++m) o[44 + m] = C.jac[m];
            o[60] = tau;
        } else {
            set_status(B.status, ST_NONFINITE_FLUX);
        }
    }
}

// ugks_node's flux at one face Gauss node (mod_S2D1.f90:486-507): one CTA per (face, node), VPT
// velocities per thread, from the node scalars; the node micro flux goes to SB.node, its moments to
// SB.nodew, and the time-direction moment gate (2e-12) is checked on the block-reduced moments.
// Three CTAs per SM (80 registers, small spills): the kernel waits on its face-cache loads, and 24
// resident warps hide that better than 16.
template <int VPT>
__global__ void __launch_bounds__(256, 3) k_s2_face_flux(LoParams P, LoBuffers B, S2Buffers SB) {
    if (eval_cached(B)) return;
    __shared__ double sc[kS2FScal];
    __shared__ double red[8 * 8];
    __shared__ double rout[kRedSlots];
    const int nv = P.nvel, nx = P.nx, ny = P.ny, ck = P.ck;
    const int nfx = nx * ny;
    const int wid = blockIdx.x, fi = wid / 3, g = wid % 3;
    const int axis = fi < nfx ? 0 : 1, f = axis == 0 ? fi : fi - nfx;
    const int cl = f, i = cl % nx, j = cl / nx;
    const int cr = axis == 0 ? j * nx + (i + 1) % nx : (j + 1) * nx + i;
    if (threadIdx.x < kS2FScal) sc[threadIdx.x] = SB.fscal[(size_t)wid * kS2FScal + threadIdx.x];
    __syncthreads();
    if (sc[0] == 0.0) return;   // the scalars kernel failed (status set there)
    double th[4], tdl[4], tdr[4], tdt[4], tdm[4], mt[5];
    WMke M;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        th[m] = sc[1 + m]; M.tdx[m] = sc[5 + m]; M.tdy[m] = sc[9 + m];
        tdl[m] = sc[19 + m]; tdr[m] = sc[23 + m]; tdt[m] = sc[27 + m]; tdm[m] = sc[31 + m];
    }
    M.ux = sc[13]; M.vy = sc[14]; M.lam = sc[15]; M.coeff = sc[16];
    const double q0x = sc[17], q0y = sc[18];
#pragma unroll
    for (int m = 0; m < 5; ++m) mt[m] = sc[35 + m];
    const S2Th tt = s2_th(th, ck);
    double* outh = SB.node + (size_t)wid * 2 * nv;
    double* outb = outh + nv;
    double acc[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) acc[m] = 0.0;
    int bad = 0;
#pragma unroll
    for (int r = 0; r < VPT; ++r) {
        const Slot sl_ = slot(r, nv);
        const int k = sl_.kk;
        const double uk = B.u[k], vk = B.v[k], wk = sl_.ok ? B.w[k] : 0.0;
        S2Q q;
        double mh, mb, kxh, kxb, kyh, kyb;
        w_mke_at(tt, M, ck, uk, vk, q, mh, mb, kxh, kxb, kyh, kyb);
        const double s0h = mh + kxh * q0x + kyh * q0y;
        const double s0b = mb + kxb * q0x + kyb * q0y;
        double dlh, dlb, drh, drb, dth, dtb, mth, mtb;
        s2_dq(q, tdl, dlh, dlb);
        s2_dq(q, tdr, drh, drb);
        s2_dq(q, tdt, dth, dtb);
        s2_dq(q, tdm, mth, mtb);
        moment_add(wk, uk, vk, mth, mtb, acc);
        const double vn = axis == 0 ? uk : vk, vt = axis == 0 ? vk : uk;
        const bool left = vn >= 0.0;
        const double* rc = SB.rec + rec_cell(left ? cl : cr, axis, 0, g, nv) + k;   // fields 3 nv apart
        const double f0h = rc[0], f0b = rc[(size_t)3 * nv], nh = rc[(size_t)6 * nv], th_ = rc[(size_t)9 * nv];
        const double nb = rc[(size_t)12 * nv], tb_ = rc[(size_t)15 * nv];
        const double sh = vn * (left ? dlh : drh) + vt * dth;
        const double sb = vn * (left ? dlb : drb) + vt * dtb;
        const double fhv = vn * (mt[0] * s0h + mt[1] * sh + mt[2] * mth + mt[3] * f0h - mt[4] * (vn * nh + vt * th_));
        const double fbv = vn * (mt[0] * s0b + mt[1] * sb + mt[2] * mtb + mt[3] * f0b - mt[4] * (vn * nb + vt * tb_));
        moment_add(wk, uk, vk, fhv, fbv, acc + 4);
        if (sl_.ok) {
            outh[sl_.k] = fhv;
            outb[sl_.k] = fbv;
            if (!(isfinite(fhv) && isfinite(fbv))) bad = 1;
            if (SB.coef) {   // ugks_node's f0_h, f0_b, k_h, k_b (mod_S2D1.f90:501-505)
                double* cf = SB.coef + (size_t)wid * 4 * nv + sl_.k;
                const double tau = sc[60];
                cf[0] = vn * f0h;
                cf[(size_t)nv] = vn * f0b;
                cf[2 * (size_t)nv] = vn * ((s0h - f0h) / tau - vn * nh - vt * th_);
                cf[3 * (size_t)nv] = vn * ((s0b - f0b) / tau - vn * nb - vt * tb_);
            }
        }
    }
    block_reduce_smem<8, 0>(acc, red, rout);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double mx = 0.0, scl = 1.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) { mx = fmax(mx, fabs(rout[m] - sc[40 + m])); scl = fmax(scl, fabs(sc[40 + m])); }
#pragma unroll
        for (int m = 0; m < 4; ++m) SB.nodew[(size_t)wid * 4 + m] = rout[4 + m];
        if (bad || !(mx / scl <= 2.0e-12)) set_status(B.status, ST_NONFINITE_FLUX);
    }
}

// wall face nodes (s2w2_wall_node, mod_S2MultiscaleWall.f90:45-184): one warp per (wall face,
// Gauss node); bottom faces of row 0, then top faces of row ny-1.  Node fluxes go to the node
// buffers after the interior faces.
__global__ void __launch_bounds__(256, 2) k_s2_wall_nodes(LoParams P, LoBuffers B, S2Buffers SB, int qrec) {
    if (eval_cached(B)) return;
    extern __shared__ double s_qrec[];
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
    const double wc[4] = {wcell[0], wcell[2], -wcell[1], wcell[3]};
    const double wg[4] = {prim_g[0], 0.0, -prim_g[0] * ux, prim_g[0] * ((double)(ck + 2) / (4.0 * lambda) + 0.5 * ux * ux)};
    // wall_equilibrium: the discrete closure of the wall state
    const double wwall[4] = {prim_g[0], prim_g[0] * ux, 0.0, prim_g[0] * ((double)(ck + 2) * theta / 2.0 + ux * ux / 2.0)};
    __shared__ double s_jac[8][16];
    WClosure C;
    C.jac = s_jac[threadIdx.x >> 5];
    const WQRec qr{qrec ? s_qrec + (threadIdx.x >> 5) * (nr * 32) : nullptr};
    bool ok = pp > 0.0 && isfinite(pp) && w_closure(P, B, wwall, C, qr);
    auto rec = [&](const WVel& s, int field) {
        return SB.rec[rec_wall(nx, ny, top, i, field, g, nv) + s.k];
    };
    double acc[8];
    double an[4], at[4], atime[4], mt[5], mxi2 = 0.0, coeff = 0.0, hlx = 0.0, hly = 0.0, tau_wall = 0.0;
    if (ok) {
#pragma unroll
        for (int m = 0; m < 6; ++m) acc[m] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            const double hin = rec(s, 0), bin = rec(s, 1), ht = rec(s, 3), bt = rec(s, 5);
            const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
            acc[0] += s.w * (-ht);
            acc[1] += s.w * (-(vn * ht));
            acc[2] += s.w * (-(vt * ht));
            acc[3] += s.w * (-(0.5 * (v2 * ht + bt)));
            const double vt2 = -s.u + ux, w2 = vn * vn + vt2 * vt2;
            acc[4] += 0.5 * s.w * vn * (w2 * hin + bin);
            acc[5] += 0.5 * s.w * vt2 * (w2 * hin + bin);
        }
        warp_sum_all<6>(acc);
        double sw[4], sw_t[4], Mu[7], Mv[6], Mxi[3], m1[4], m2[4];
        for (int m = 0; m < 4; ++m) { sw[m] = (wg[m] - wc[m]) / (side * 0.5 * P.dy); sw_t[m] = acc[m]; }
        s2w_micro_slope(ck, prim_g, sw, an);
        s2w_micro_slope(ck, prim_g, sw_t, at);
        s2w_moments(ck, prim_g, Mu, Mv, Mxi);
        s2w_auvxi(an, Mu, Mv, Mxi, 1, 0, m1);
        s2w_auvxi(at, Mu, Mv, Mxi, 0, 1, m2);
        for (int m = 0; m < 4; ++m) sw[m] = -prim_g[0] * (m1[m] + m2[m]);
        s2w_micro_slope(ck, prim_g, sw, atime);
        const double wgg[4] = {wg[0], -wg[2], wg[1], wg[3]};
        ok = s2_tau(P, wgg, tau_wall);
        s2w_time_coeffs(dt, tau_wall, mt);
        coeff = P.pr != 1.0 ? 0.8 * (1.0 - P.pr) * lambda * lambda / prim_g[0] : 0.0;
        mxi2 = Mxi[2];
        hlx = acc[4];
        hly = acc[5];
    }
    // the incident micro flux g_in and the reflected wall Maxwellian of one velocity
    const S2Th tt = s2_th(C.th, ck);
    auto gin = [&](const WVel& s, int r, double& ginh, double& ginb, double& wallh, double& wallb, double& mh,
                   double& mb, double& corrh, double& corrb) {
        const S2Q q = qr.at(tt, s, r);
        mh = q.qh;
        mb = q.qb;
        wallh = mh / prim_g[0];
        wallb = mb / prim_g[0];
        corrh = 0.0;
        corrb = 0.0;
        if (P.pr != 1.0) {
            const double vn = s.v, vt = -s.u + ux, v2 = vn * vn + vt * vt;
            const double qdot = vn * hlx + vt * hly, shh = 2.0 * lambda * v2 - 4.0;
            corrh = coeff * qdot * shh * mh;
            corrb = coeff * qdot * (shh + 2.0 / (double)ck) * mb;
        }
        const double vn = s.v, vt = -s.u, v2 = vn * vn + vt * vt;
        const double Han = (an[0] + an[1] * vn + an[2] * vt) * mh + 0.5 * an[3] * (v2 * mh + mb);
        const double Hatan = (at[0] + at[1] * vn + at[2] * vt) * mh + 0.5 * at[3] * (v2 * mh + mb);
        const double Hatime = (atime[0] + atime[1] * vn + atime[2] * vt) * mh + 0.5 * atime[3] * (v2 * mh + mb);
        const double Ban = (an[0] + an[1] * vn + an[2] * vt) * mb + 0.5 * an[3] * (v2 * mb + mxi2 * mh);
        const double Batan = (at[0] + at[1] * vn + at[2] * vt) * mb + 0.5 * at[3] * (v2 * mb + mxi2 * mh);
        const double Batime = (atime[0] + atime[1] * vn + atime[2] * vt) * mb + 0.5 * atime[3] * (v2 * mb + mxi2 * mh);
        ginh = mt[0] * mh + mt[1] * (vn * Han + vt * Hatan) + mt[2] * Hatime + mt[3] * rec(s, 0) -
               mt[4] * (vn * rec(s, 2) + s.u * rec(s, 3));
        ginb = mt[0] * mb + mt[1] * (vn * Ban + vt * Batan) + mt[2] * Batime + mt[3] * rec(s, 1) -
               mt[4] * (vn * rec(s, 4) + s.u * rec(s, 5));
        ginh = ginh + mt[0] * corrh;
        ginb = ginb + mt[0] * corrb;
    };
    double inc = 0.0, rhow = 0.0;
    if (ok) {   // incidence and reflection -> wall density
        acc[0] = acc[1] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb, mh, mb, ch, cb;
            gin(s, r, ginh, ginb, wallh, wallb, mh, mb, ch, cb);
            if (side * s.v > 0.0) acc[0] += s.w * s.v * ginh;
            else acc[1] += dt * s.w * s.v * wallh;
        }
        warp_sum_all<2>(acc);
        inc = acc[0];
        const double refl = acc[1];
        rhow = -inc / refl;
        ok = isfinite(refl) && fabs(refl) > DBL_MIN && isfinite(rhow) && rhow > 0.0;
    }
    if (ok) {
        double* outh = SB.node + node * 2 * nv;
        double* outb = outh + nv;
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[m] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb, mh, mb, ch, cb, fh, fb;
            gin(s, r, ginh, ginb, wallh, wallb, mh, mb, ch, cb);
            if (side * s.v > 0.0) { fh = s.v * ginh; fb = s.v * ginb; }
            else { fh = dt * s.v * rhow * wallh; fb = dt * s.v * rhow * wallb; }
            acc[0] += s.w * fh; acc[1] += s.w * (s.u * fh); acc[2] += s.w * (s.v * fh);
            acc[3] += s.w * (0.5 * ((s.u * s.u + s.v * s.v) * fh + fb));
            if (s.ok) {
                outh[s.k] = fh;
                outb[s.k] = fb;
                ok = ok && isfinite(fh) && isfinite(fb);
            }
        }
        warp_sum_all<4>(acc);
        ok = ok && isfinite(acc[0]) && fabs(acc[0]) <= 2.0e-12 * fmax(1.0, fabs(inc));
        if (lane < 4) SB.nodew[node * 4 + lane] = lane == 0 ? acc[0] : (lane == 1 ? acc[1] : (lane == 2 ? acc[2] : acc[3]));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (ok && SB.coef) {   // the optional f0_h, f0_b, k_h, k_b outputs (mod_S2MultiscaleWall.f90:155-177)
        auto qk = [&](const WVel& s, double m, double corr, int fv, int fn, int ft) {
            return (m + corr - rec(s, fv)) / tau_wall - s.v * rec(s, fn) - s.u * rec(s, ft);
        };
        acc[0] = acc[1] = acc[2] = 0.0;
        for (int r = 0; r < nr; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb, mh, mb, ch, cb;
            gin(s, r, ginh, ginb, wallh, wallb, mh, mb, ch, cb);
            if (side * s.v > 0.0) {
                acc[0] += s.w * s.v * rec(s, 0);
                acc[1] += s.w * s.v * qk(s, mh, ch, 0, 2, 3);
            } else {
                acc[2] += s.w * s.v * wallh;
            }
        }
        warp_sum_all<3>(acc);
        const double r0 = -acc[0] / acc[2], r1 = -acc[1] / acc[2];
        ok = isfinite(r0) && isfinite(r1) && r0 > 0.0;
        double* cf = SB.coef + node * 4 * nv;
        acc[0] = acc[1] = 0.0;
        for (int r = 0; r < nr && ok; ++r) {
            const WVel s = wvel(B, nv, r);
            double ginh, ginb, wallh, wallb, mh, mb, ch, cb, c0, c1, c2, c3;
            gin(s, r, ginh, ginb, wallh, wallb, mh, mb, ch, cb);
            if (side * s.v > 0.0) {
                c0 = s.v * rec(s, 0);
                c1 = s.v * rec(s, 1);
                c2 = s.v * qk(s, mh, ch, 0, 2, 3);
                c3 = s.v * qk(s, mb, cb, 1, 4, 5);
            } else {
                c0 = s.v * r0 * wallh;
                c1 = s.v * r0 * wallb;
                c2 = s.v * r1 * wallh;
                c3 = s.v * r1 * wallb;
            }
            acc[0] += s.w * c0;
            acc[1] += s.w * c2;
            if (s.ok) {
                cf[s.k] = c0;
                cf[(size_t)nv + s.k] = c1;
                cf[2 * (size_t)nv + s.k] = c2;
                cf[3 * (size_t)nv + s.k] = c3;
            }
        }
        if (ok) {
            warp_sum_all<2>(acc);
            ok = fabs(acc[0]) <= 2.0e-12 && fabs(acc[1]) <= 2.0e-12;
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) set_status(B.status, ST_NONFINITE_FLUX);
}

// Gauss-weighted sum of the node fluxes of every face (interior, then the walls) times the face
// length, into the face arrays ComputeResidual reads; the walls' macro fluxes also unscaled into
// SB.wall_raw, and the walls' (pnn, pnt, qn) into B.wall_aero.  One thread per (face, velocity);
// threads k < 4 also do the macro flux.
__global__ void __launch_bounds__(256) k_s2_combine(LoParams P, LoBuffers B, S2Buffers SB, int f0) {
    if (eval_cached(B)) return;
    const int nv = P.nvel, nx = P.nx, ny = P.ny, nfx = nx * ny, nf = nfx + nx * (ny - 1);
    const int fi = f0 + (int)blockIdx.y;
    const int k = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= nv) return;
    const double gw[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
    size_t o;
    double len, *Fh, *Fb, *Fw;
    int wall = -1;
    if (fi < nfx) {
        const int i = fi % nx, j = fi / nx;
        o = (size_t)j * nx + (i + 1) % nx; len = P.dy; Fh = B.fxh; Fb = B.fxb; Fw = B.fxw;
    } else if (fi < nf) {
        const int f = fi - nfx, i = f % nx, j = f / nx;
        o = (size_t)(j + 1) * nx + i; len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    } else {
        wall = fi - nf;
        const int top = wall >= nx ? 1 : 0, i = wall - top * nx;
        o = top ? (size_t)ny * nx + i : (size_t)i; len = P.dx; Fh = B.fyh; Fb = B.fyb; Fw = B.fyw;
    }
    const double* nd = SB.node + (size_t)fi * 3 * 2 * nv;
    double afh = 0.0, afb = 0.0;
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        afh = afh + gw[g] * nd[(size_t)(2 * g) * nv + k];
        afb = afb + gw[g] * nd[(size_t)(2 * g + 1) * nv + k];
    }
    Fh[o * nv + k] = afh * len;
    Fb[o * nv + k] = afb * len;
    if (k < 4) {
        double afw = 0.0;
#pragma unroll
        for (int g = 0; g < 3; ++g) afw = afw + gw[g] * SB.nodew[((size_t)fi * 3 + g) * 4 + k];
        Fw[o * 4 + k] = afw * len;
        if (wall >= 0 && SB.wall_raw != nullptr) SB.wall_raw[(size_t)wall * 4 + k] = afw;
    }
    if (wall >= 0 && k == 0) {   // PublishWallDiagnostics (mod_S2NativeAdapter.f90:1075-1097)
        const int top = wall >= nx ? 1 : 0;
        const double measure = B.dt[0] * len;
        double rate[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double afw = 0.0;
#pragma unroll
            for (int g = 0; g < 3; ++g) afw = afw + gw[g] * SB.nodew[((size_t)fi * 3 + g) * 4 + m];
            rate[m] = afw * len / measure;
        }
        // native frame n = +y, t = -x; the heat removes the moving wall's mechanical work
        double* a = B.wall_aero + (size_t)wall * 3;
        a[0] = rate[2];
        a[1] = -rate[1];
        a[2] = rate[3] - P.wall_ux[top] * rate[1];
    }
}


// Shared memory for the closure kernels' Maxwellian records (WQRec): one record of the velocity set
// per warp, used when it fits these caps.  The caps keep the kernels' resident CTAs per SM: three
// 128-thread face-node CTAs (up to 2304 = 48^2 velocities), two 256-thread target- and face-node CTAs
// (up to 1760 velocities).  The wall-node kernel has only 6 nx warps: one CTA per SM will do.
constexpr int kQRecCap128x3 = 72 * 1024, kQRecCap256x2 = 110 * 1024, kQRecCapWall = 200 * 1024;

cudaError_t prepare_s2() {
    cudaError_t e = s2_upload_tables();
    const auto dyn = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_s2_face_nodes<kS2NodeThreads, 3>, dyn, kQRecCap128x3);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_s2_face_nodes<256, 2>, dyn, kQRecCap256x2);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_s2_target_nodes, dyn, kQRecCap256x2);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_s2_wall_nodes, dyn, kQRecCapWall);
    return e;
}

// bytes of the Maxwellian records of a CTA of `threads` threads, 0 (no records) above `cap`.  Many
// instances on concurrent streams (S2Buffers::concurrent) take none: their kernels share SMs with other
// instances' kernels, and the records' shared-memory carve-out cost the batch more than it saved it
// (7.47e8 -> 7.44e8 updates/s for the 256-instance distribution, same GPU); the values are the same
// either way.
static int qrec_bytes(const S2Buffers& S, int nv, int threads, int cap) {
    const long long b = (long long)(threads / 32) * ((nv + 31) / 32) * 32 * (long long)sizeof(double);
    return !S.concurrent && b <= cap ? (int)b : 0;
}


// which 0: the S2 cold start; 1: the S2 Evolution of one pseudo-step (targets, reconstruction,
// faces, walls); 2: the Evolution with the targets kept (S2CN2); 3: the targets of B.W only
cudaError_t s2_enqueue(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                       cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    const int nx = P.nx, ny = P.ny, nv = P.nvel, nc = nx * ny, nf = nx * ny + nx * (ny - 1);
    auto warps = [](long long n) { return (unsigned)((n * 32 + 255) / 256); };
    auto node_ctas = [](long long n) { return (unsigned)((n * 32 + kS2NodeThreads - 1) / kS2NodeThreads); };
    if (which == 0) {
        k_s2_init<<<warps(nc), 256, 0, s>>>(P, B, S);
        return cudaGetLastError();
    }
    if (which == 4) {
        const dim3 grid((unsigned)((nv + 31) / 32), (unsigned)nc);
        k_s2_recon1<<<grid, 128, 0, s>>>(P, B, S);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) { k_s2_recon2<<<grid, 256, 0, s>>>(P, B, S); e = cudaGetLastError(); }
        return e;
    }
    const int faces = which != 3, targets = which != 2;
    const long long nmacw = (faces ? (long long)nf * 2 : 0) + (targets ? (long long)nc : 0);   // warps
    k_s2_macro<<<(unsigned)((nmacw * 32 + 127) / 128), 128, 0, s>>>(P, B, S, faces, targets);
    cudaError_t e = cudaGetLastError();
    // which 1: the targets need only the macro pass and are first read after the face combine, so
    // they run on the side stream beside the reconstruction and the face nodes (the wall nodes
    // follow them there); which 3: on the main stream
    const bool side_targets = targets && faces;
    if (e == cudaSuccess && side_targets) {
        e = cudaEventRecord(fork, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    }
    if (e == cudaSuccess && targets) {
        cudaStream_t ts = side_targets ? s2 : s;
        const int qb = qrec_bytes(S, nv, 256, kQRecCap256x2);
        k_s2_target_nodes<<<warps((long long)nc * 9), 256, qb, ts>>>(P, B, S, qb > 0);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            k_s2_target_sum<<<dim3((unsigned)((nv + 255) / 256), (unsigned)nc), 256, 0, ts>>>(P, B, S);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess || which == 3) return e;
    const dim3 grid((unsigned)((nv + 31) / 32), (unsigned)nc);
    k_s2_recon1<<<grid, 128, 0, s>>>(P, B, S);
    e = cudaGetLastError();
    if (e == cudaSuccess) { k_s2_recon2<<<grid, 256, 0, s>>>(P, B, S); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cudaEventRecord(fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, fork, 0);
    if (e == cudaSuccess) {
        if (P.s2_kinetic) e = launch_s2_w1_walls(P, B, S, s2);
        else {
            const int qb = qrec_bytes(S, nv, 256, kQRecCapWall);
            k_s2_wall_nodes<<<warps(2LL * nx * 3), 256, qb, s2>>>(P, B, S, qb > 0);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(join, s2);
    if (e == cudaSuccess) {
        if (S.concurrent) {
            const int qb = qrec_bytes(S, nv, 256, kQRecCap256x2);
            k_s2_face_nodes<256, 2><<<warps((long long)nf * 3), 256, qb, s>>>(P, B, S, qb > 0);
        } else {
            const int qb = qrec_bytes(S, nv, kS2NodeThreads, kQRecCap128x3);
            k_s2_face_nodes<kS2NodeThreads, 3><<<node_ctas((long long)nf * 3), kS2NodeThreads, qb, s>>>(P, B, S, qb > 0);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        if (nv <= 1024) k_s2_face_flux<4><<<(unsigned)(nf * 3), 256, 0, s>>>(P, B, S);
        else k_s2_face_flux<10><<<(unsigned)(nf * 3), 256, 0, s>>>(P, B, S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, join, 0);
    if (e == cudaSuccess) e = launch_s2_combine(P, B, S, 0, nf + 2 * nx, s);
    return e;
}

cudaError_t launch_s2_combine(const LoParams& P, const LoBuffers& B, const S2Buffers& S, int f0, int nfaces,
                              cudaStream_t s) {
    k_s2_combine<<<dim3((unsigned)((P.nvel + 255) / 256), (unsigned)nfaces), 256, 0, s>>>(P, B, S, f0);
    return cudaGetLastError();
}

}  // namespace ugks
