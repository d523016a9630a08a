// ugks_s2.cuh -- device state of the high-order S2 evolution (HighOrderImplicit).
#pragma once
#include "ugks_lo.cuh"

namespace ugks {

// WENO-AO(5,3) reconstruction maps (mod_S2D1Reconstruction.f90:57-111), built on the host with the
// reference's own small solve: cmap[c][k][d] = coefficient of xi^d contributed by sample k of
// candidate c; wall[side][distance-1][k][d] the one-sided quartic; gnode the 3 Gauss nodes.
struct S2Maps {
    double cmap[4][5][5];
    double wall[2][3][5][5];
    double gnode[3];
};

// The face cache (S2Buffers::rec): the limited face values and normal / tangential derivatives of h and b
// (fields 0..5: h, b, h_n, h_t, b_n, b_t) at the 3 Gauss nodes of a cell's sides.  Per velocity a cell
// keeps, along each axis, only the side that velocity leaves it through (x: the right side when u >= 0,
// else the left; y: the top when v >= 0, else the bottom) -- the upwind side, the only one an interior face
// reads: [cell][axis][field][node][nvel].  The wall rows' wall sides follow for every velocity (the wall
// node reads both halves): [wall: bottom, top][i][field][node][nvel].
__host__ __device__ __forceinline__ size_t s2_rec_doubles(int nx, int ny, int nv) {
    return ((size_t)nx * ny * 36 + (size_t)2 * nx * 18) * (size_t)nv;
}
__host__ __device__ __forceinline__ size_t rec_cell(int cell, int axis, int field, int node, int nv) {
    return ((((size_t)cell * 2 + axis) * 6 + field) * 3 + node) * (size_t)nv;
}
__host__ __device__ __forceinline__ size_t rec_wall(int nx, int ny, int wall, int i, int field, int node, int nv) {
    return ((size_t)nx * ny * 36 + (((size_t)wall * nx + i) * 6 + field) * 3 + node) * (size_t)nv;
}
// whether velocity (u, v) leaves a cell through side p (0 x left, 1 x right, 2 y bottom, 3 y top): the
// upwind selector of the faces, vn >= 0 taking the lower cell's upper side
__host__ __device__ __forceinline__ bool rec_leaves(int p, double u, double v) {
    const bool hi = (p < 2 ? u : v) >= 0.0;
    return (p & 1) ? hi : !hi;
}

struct S2Buffers {
    double* rec;                        // the face cache (layout above, s2_rec_doubles)
    double *mh, *mb, *kxh, *kxb, *kyh, *kyb;   // [cell][nvel] volume targets
    double* wall_raw;                   // [2][nx][4] wall macro fluxes before the face length (bottom,
                                        // top), for the S2CN2 conservation ledger (nullptr: not kept)
    // evaluation scratch (s2_bind_scratch)
    double* node;    // [face][3 nodes][h | b][nvel] Gauss-node micro fluxes; faces: interior x, interior y, walls
    double* nodew;   // [face][3][4] Gauss-node macro fluxes
    double* mac;     // [interior face][3][normal left | normal right | tangential][4] macro slopes
    double* wq;      // [cell][9][4] mean-shifted volume node states
    double* tscal;   // [cell][9][16] volume node scalars (closure theta, directions, primitive)
    double* l1;      // [cell][22][nvel] first-layer WENO values of h and b (k_s2_recon1)
    double* fscal;   // [interior face][3][kS2FScal] face-node scalars (k_s2_face_nodes -> k_s2_face_flux)
    double* coef;    // [face node][f0 h, f0 b, k h, k b][nvel] the leading and time coefficients of every node
                     // flux (ugks_node's and s2w2_wall_node's optional outputs) for the wall variants that
                     // correct the faces; nodes as `node` (nullptr: not wanted)
    int concurrent;  // 1: one of many instances on concurrent streams (the batch): the closure kernels
                     // take the CTA shape with more resident warps
};

// Node scalar records.  Volume target nodes (tscal): [0..3] closure theta, [4..11] the K_x, K_y
// closure directions, [12..15] ux vy lam coeff, [16..31] the closure's moment Jacobian (row-major).
// Interior face nodes (fscal): [0] ok, [1..4] theta, [5..12] K directions, [13..16] ux vy lam coeff,
// [17..18] q0, [19..34] left/right/tangential/time directions, [35..39] Mt, [40..43] the time-direction
// moments wt, [44..59] the closure's moment Jacobian, [60] the face tau.  The Jacobians serve the adjoint (ugks_s2_adjoint.cu).
constexpr int kS2TScal = 32;
constexpr int kS2FScal = 64;

// doubles of evaluation scratch one S2Buffers needs, and their layout
inline size_t s2_scratch_doubles(int nx, int ny, int nv) {
    const size_t nf = (size_t)nx * ny + (size_t)nx * (ny - 1), nfw = nf + 2 * (size_t)nx, nc = (size_t)nx * ny;
    auto r = [](size_t n) { return (n + 31) / 32 * 32; };
    return r(nfw * 3 * 2 * nv) + r(nfw * 3 * 4) + r(nf * 3 * 12) + r(nc * 9 * 4) + r(nc * 9 * kS2TScal) + r(nc * 22 * nv) + r(nf * 3 * kS2FScal);
}
inline void s2_bind_scratch(S2Buffers& S, double* base, int nx, int ny, int nv) {
    const size_t nf = (size_t)nx * ny + (size_t)nx * (ny - 1), nfw = nf + 2 * (size_t)nx, nc = (size_t)nx * ny;
    auto r = [](size_t n) { return (n + 31) / 32 * 32; };
    S.node = base; base += r(nfw * 3 * 2 * nv);
    S.nodew = base; base += r(nfw * 3 * 4);
    S.mac = base; base += r(nf * 3 * 12);
    S.wq = base; base += r(nc * 9 * 4);
    S.tscal = base; base += r(nc * 9 * kS2TScal);
    S.l1 = base; base += r(nc * 22 * nv);
    S.fscal = base;
}

// s2_tau (mod_S2PhysicalGas.f90:9-20): GetTau of (rho, U, V, 0.5 rho / p), p = 2/(ck+2) e
__device__ __forceinline__ bool s2_tau(const LoParams& P, const double w[4], double& tau) {
    const double pr = 2.0 / (double)(P.ck + 2) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    const Prim p{w[0], w[1] / w[0], w[2] / w[0], 0.5 * w[0] / pr};
    return get_tau(P.mu_ref, P.omega, p, tau);
}

// mod_S2D1.f90 primitive (:66-79): theta_gas = p / rho
__device__ __forceinline__ bool s2_primitive(const double w[4], int ck, double& rho, double& ux, double& vy,
                                             double& th) {
    rho = w[0];
    if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3])) || w[0] <= 0.0) return false;
    ux = w[1] / w[0];
    vy = w[2] / w[0];
    const double eint = w[3] - 0.5 * w[0] * (ux * ux + vy * vy);
    if (eint <= 0.0) return false;
    const double p = (2.0 / (double)(ck + 2)) * eint;
    th = p / w[0];
    return isfinite(th) && th > 0.0;
}

cudaError_t prepare_s2();
// which 0: S2 cold start (h, b := discrete closure Maxwellian of W); 1: S2 Evolution (targets of B.W,
// reconstruction, faces, walls); 2: S2 Evolution with the targets in S kept; 3: targets of B.W into S;
// 4: the reconstruction of B's h, b into S.rec only
cudaError_t s2_enqueue(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                       cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join);
// kernels s2_enqueue(which, ...) launches: the cold start 1; the macro pass, then 2 for the targets
// (volume nodes, sum) and 6 for the evolution (reconstruction x2, wall nodes, face nodes, face flux,
// combine); the reconstruction alone 2
constexpr int s2_enqueue_kernels(int which) {
    return which == 0 ? 1 : which == 4 ? 2 : 1 + (which != 2 ? 2 : 0) + (which != 3 ? 6 : 0);
}
// the wall nodes of the kinetic (FluxWall_type 0) wall into S.node / S.nodew (ugks_s2_walls.cu)
cudaError_t launch_s2_w1_walls(const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s);
// k_s2_combine over faces [f0, f0 + nfaces) of the face numbering (interior x, interior y, walls)
cudaError_t launch_s2_combine(const LoParams& P, const LoBuffers& B, const S2Buffers& S, int f0, int nfaces,
                              cudaStream_t s);

}  // namespace ugks
