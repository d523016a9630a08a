// ugks_s2_adjoint.cuh -- the discrete adjoint (reverse mode) of one S2CN2 step.
//
// The step maps the state x = (h, b, W) and the volume targets T = targets(W) to x' and T' and, in its
// evaluation, gives the walls' shear and heat flux (PublishWallDiagnostics,
// mod_S2NativeAdapter.f90:1075-1097).  Its adjoint maps the cotangents of (x', T') and of those wall
// outputs back to cotangents of (x, T) and of the parameters mu_ref (the tau / Kn scale), the wall
// speeds and the wall temperatures.  The step's own kernels are run first on x (the forward re-run
// of the checkpoint-and-recompute schedule): the adjoint kernels read what they leave in the scratch
// (the face cache, the first layer, the node scalars, the stream state and the CN right-hand side,
// the targets of the stream state).
#pragma once
#include "ugks_s2cn2.cuh"

namespace ugks {

// parameter cotangents (AdjBuffers::gpar): d/d mu_ref, d/d wall_ux[0..1], d/d wall_tnative[0..1]
enum { GP_MU = 0, GP_UX0 = 1, GP_UX1 = 2, GP_TW0 = 3, GP_TW1 = 4, GP_COUNT = 8 };

struct AdjBuffers {
    // cotangents of the step's outputs: x' = (h', b', W') and T' = targets(W'); gTo accumulates (the
    // later step's stream adjoint wrote it, this step's collision adds to it)
    double *gho, *gbo, *gWo;
    double* gTo[6];          // mh, mb, kxh, kxb, kyh, kyb
    // cotangents of the step's inputs (written by this step)
    double *ghi, *gbi, *gWi;
    double* gTi[6];
    // intermediates of one step
    double *grh, *grb;       // [nc][nvel] the CN right-hand side
    double* gws;             // [nc][4]    the stream state (= W')
    double* gwq;             // [nc][9][4] the volume node states of the stream state
    double* grec;            // [nc][72][nvel] the face cache
    double* gl1;             // [nc][22][nvel] the first layer (zeroed by its consumer)
    double* gmac;            // [interior face][3][12] the macro slopes
    double* gpar;            // [GP_COUNT] parameter cotangents, accumulated over the steps
    const double* seed;      // [4] cotangents of (bottom shear, bottom heat, top shear, top heat) of this
                             // step's evaluation, or nullptr
    unsigned* status;        // [1] the adjoint's own status word (ST_ADJOINT_DT); the forward's stays clean so
                             // that the forward re-runs never halt on an adjoint check
};

constexpr unsigned ST_ADJOINT_DT = 1u << 10;   // the constant-dt assumption of the adjoint does not hold

// doubles of adjoint work one instance needs (AdjBuffers minus the four cotangent state sets)
size_t adj_work_doubles(int nx, int ny, int nv);
void adj_bind_work(AdjBuffers& A, double* base, int nx, int ny, int nv);

cudaError_t prepare_s2_adjoint();

// The adjoint of one step whose forward re-run has just filled S (evaluation scratch), C (stream state,
// CN right-hand side) and To (targets of the stream state, with their node scalars in S):
// x = (B.h, B.b, B.W), T = targets of B.W.  Reads A.gho .. A.gTo, writes A.ghi .. A.gTi and adds to
// A.gpar.  Launches on s; with s2 and ev (4 events) the wall nodes and the macro slopes' transpose run on
// s2 beside the interior face nodes and recon2, and s has waited for s2 when the call returns.
cudaError_t enqueue_s2cn2_adjoint(const LoParams& P, const LoBuffers& B, const S2Buffers& S, const S2Buffers& T,
                                  const S2Buffers& To, const CnBuffers& C, const AdjBuffers& A, cudaStream_t s,
                                  cudaStream_t s2 = nullptr, const cudaEvent_t* ev = nullptr);
// The targets adjoint alone: the cotangent gT of targets(W) (with W's node scalars in S, just built by
// s2_enqueue(3)) added to gW.
cudaError_t enqueue_targets_adjoint(const LoParams& P, const LoBuffers& B, const S2Buffers& S, double* const gT[6],
                                    double* gW, const AdjBuffers& A, cudaStream_t s);
constexpr int kAdjStepKernels = 10;

}  // namespace ugks
