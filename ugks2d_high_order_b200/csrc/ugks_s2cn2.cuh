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
    int predict;         // 1: the CN collision of a predictor (the W1T midpoint): its gates only, no report,
                         // ledger or acceptance; a failure stops the step with ST_W1T_PREDICTOR
};

// The research S2CN2 wall variants' own buffers (ugks_s2_walls.cu): the W1T midpoint predictor's half dt,
// face arrays, evaluation set and stream state; the predicted state; W2R's instantaneous wall node fluxes.
struct CnVariant {
    double* half;                                // [2] dt/2 of the step
    double *fxh, *fxb, *fxw, *fyh, *fyb, *fyw;   // the predictor's face arrays (LoBuffers layout)
    double* wall_aero;                           // [2][nx][3] the predictor's wall diagnostics (unused)
    S2Buffers Sp;                                // face cache, evaluation scratch, targets of the predicted state
    CnBuffers Cp;                                // stream state, CN right-hand side, cell diagnostics (predict = 1)
    double *h, *b, *W;                           // the predicted state
    double* inst;                                // [2 nx][3][h | b][nvel] instantaneous wall node fluxes (W2R)
};
// the variant's part of a step after the official evaluation and before k_cn_stream, and the kernels
// it launches
cudaError_t enqueue_s2cn2_variant(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const CnVariant& V,
                                  cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join);
int s2cn2_variant_kernels(const LoParams& P);

// One S2CN2 step from state set (B, T) into state set (Bo, To); see ugks_s2cn2.cu.  V: the wall variant's
// buffers when P names a variant (nullptr otherwise).  timestep = false: the step's dt is the one its
// predecessor's k_cn_collide took from the state it accepted (steps of one sequence after its first).
cudaError_t enqueue_s2cn2_step(const LoParams& P, const LoBuffers& B, const S2Buffers& T, const LoBuffers& Bo,
                               const S2Buffers& To, const CnBuffers& C, cudaStream_t s, cudaStream_t s2,
                               cudaEvent_t fork, cudaEvent_t join, long long* launches,
                               const CnVariant* V = nullptr, bool timestep = true);
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
