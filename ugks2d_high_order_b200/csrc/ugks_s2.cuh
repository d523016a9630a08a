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

struct S2Buffers {
    double* rec;                        // [cell][72][nvel] limited face values / derivatives
    double *mh, *mb, *kxh, *kxb, *kyh, *kyb;   // [cell][nvel] volume targets
};

// s2_tau (mod_S2PhysicalGas.f90:9-20): GetTau of (rho, U, V, 0.5 rho / p), p = 2/(ck+2) e
__device__ __forceinline__ bool s2_tau(const LoParams& P, const double w[4], double& tau) {
    const double pr = 2.0 / (double)(P.ck + 2) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0]);
    const Prim p{w[0], w[1] / w[0], w[2] / w[0], 0.5 * w[0] / pr};
    return get_tau(P.mu_ref, P.omega, p, tau);
}

cudaError_t prepare_s2();
// which 0: S2 cold start (h, b := discrete closure Maxwellian of W); 1: S2 Evolution
cudaError_t s2_enqueue(int which, const LoParams& P, const LoBuffers& B, const S2Buffers& S, cudaStream_t s,
                       cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join);

}  // namespace ugks
