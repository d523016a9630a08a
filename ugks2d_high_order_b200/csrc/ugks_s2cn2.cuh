// ugks_s2cn2.cuh -- device state of the explicit high-order S2CN2 step.
#pragma once
#include "ugks_s2.cuh"

namespace ugks {

constexpr int kCnCell = 8;     // per-cell advance diagnostics
constexpr int kCnReport = 24;  // report of the last step (layout at enqueue_s2cn2_step)
// kernels of one S2CN2 step: timestep, the evolution keeping the targets, k_cn_stream, the targets of
// the stream state, k_cn_collide
constexpr int kCnStepKernels = 1 + s2_enqueue_kernels(2) + 1 + s2_enqueue_kernels(3) + 1;
static_assert(kCnStepKernels == 13, "one S2CN2 step launches 13 kernels");

struct CnBuffers {
    double* ws;          // [nc][4]    stream state W + res_w (the proposal's W)
    double* rh;          // [nc][nvel] CN right-hand side hs + beta_old (M + K q_old - h)
    double* rb;
    double* cell;        // [nc][kCnCell] per-cell: max 2 beta, cnres, mmerr, min/max h, min/max b, nonfinite
    double* ledger;      // [9] total0[4], cumulative wall balance[4], [8] step of this sequence whose
                         // conservation gate is forced to fail (0: none)
    double* report;      // [kCnReport]
    const double* wall_raw;   // [2][nx][4] this step's wall macro fluxes (written by the wall kernel)
    unsigned* halt;      // [1] set by a rejected step; every later kernel of the sequence returns at entry
    unsigned* counter;   // [1] last-CTA counter (self-resetting)
    unsigned* accepted;  // [1] accepted steps since the caller last cleared it
};

// One S2CN2 step from state set (B, T) into state set (Bo, To); see ugks_s2cn2.cu.
cudaError_t enqueue_s2cn2_step(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const LoBuffers& Bo,
                               const S2Buffers& To, const CnBuffers& C, cudaStream_t s, cudaStream_t s2,
                               cudaEvent_t fork, cudaEvent_t join, long long* launches);
// The two halves of the step after the evolution, for the per-operator C ABI (ComputeResidual, then
// S2NativeApplyUpdate): k_cn_stream of set (B, T); then the targets of the stream state into To and
// k_cn_collide into Bo with the acceptance.  enqueue_s2cn2_step launches exactly these.
cudaError_t enqueue_cn_stream(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnBuffers& C,
                              cudaStream_t s);
cudaError_t enqueue_cn_apply(const LoParams& P, const LoBuffers& B, const LoBuffers& Bo, const S2Buffers& To,
                             const CnBuffers& C, cudaStream_t s);
// S2NativeInitializeState's ledger of the state in B (total0 = sum of W, empty wall balance) and the
// volume targets of that state into T.
cudaError_t enqueue_s2cn2_prepare(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnBuffers& C,
                                  cudaStream_t s, long long* launches);

}  // namespace ugks
