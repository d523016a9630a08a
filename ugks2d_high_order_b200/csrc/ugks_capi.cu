// ugks_capi.cu -- C ABI (include/ugks_b200.h): context, device buffers, launch sequencing,
// CUDA-graph replay of the explicit step, status mapping and kernel timing.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/ugks_b200.h"
#include "ugks_implicit.cuh"
#include "ugks_s2_adjoint.cuh"
#include "ugks_s2cn2.cuh"

namespace ugks {
int lo_threads(int nvel);
cudaError_t launch_lo_slopes(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_faces(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_walls(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_cells(const LoParams& P, const LoBuffers& B, int mode, bool collision, cudaStream_t s);
cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_macro_fields(const LoParams& P, const LoBuffers& B, double* out, cudaStream_t s);
cudaError_t launch_lo_init(const LoParams& P, const LoBuffers& B, double rho, double U, double V, double tn,
                           cudaStream_t s);
cudaError_t launch_im_init(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                           cudaStream_t s);
cudaError_t prepare_implicit(const LoParams& P, const ImParams& Q);
cudaError_t enqueue_implicit_step(const LoParams& P, const LoBuffers& B, const ImParams& Q, const ImBuffers& I,
                                  cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join,
                                  long long* launches, cudaEvent_t* marks, const ImCapture* cond = nullptr);
}  // namespace ugks

using namespace ugks;

struct KernelTimer {
    double total_ms = 0.0;
    long long launches = 0;
};

struct ugks_ctx {
    ugks_params prm;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;          // side stream: wall faces run beside the interior faces
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    LoParams P{};
    LoBuffers B{};
    double* dmem = nullptr;      // one allocation backing every double buffer
    unsigned* dflags = nullptr;  // [0] counter, [1] status
    size_t ndoubles = 0;
    unsigned last_status = 0;
    long long launches = 0;
    // explicit-step graph
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // ImplicitSteady
    ImParams Q{};
    ImBuffers I{};
    double* imem = nullptr;
    unsigned* iflags = nullptr;
    bool implicit_ready = false;
    cudaGraphExec_t igraph = nullptr;
    int igraph_steps = 0;
    long long igraph_launches = 0;
    ImCapture icap{};                          // body capture of the conditional pre-update evaluation
    double* hstate = nullptr;                  // pinned [2][IS_COUNT]: the state after each graph batch
    cudaEvent_t rb_ev[2] = {nullptr, nullptr};  // its copy has landed
    cudaGraphExec_t iloop = nullptr;           // WHILE node over the batch graph: the device runs the batches
    unsigned* iloop_ctr = nullptr;             // device: batches the WHILE node may still run
    long long iloop_launches = 0;              // kernels per loop iteration
    bool iloop_unavailable = false;            // its build failed: the host pipeline runs the batches
    // profiling
    int profile = 0;                           // 1: stage events, un-graphed steps; 2: stage events in the graphs
    cudaGraphExec_t pgraph = nullptr;          // profile 2: the batch graph with the stage events captured
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    KernelTimer t_slopes, t_faces, t_walls, t_cells;
    cudaEvent_t im_ev[kImStages + 1] = {};
    KernelTimer im_t[kImStages];
    // S2CN2: double-buffered state (set 0 is B's h, b, W) and volume targets
    double* cmem = nullptr;
    unsigned* cflags = nullptr;    // [0] halt, [1] last-CTA counter, [2] accepted steps
    CnBuffers C{};
    S2Buffers T[2] = {};
    LoBuffers Bs[2] = {};          // state sets 0 and 1 with the halt flag
    bool cn_ready = false;         // ledger and targets of the current state are in place
    int cn_reject_at = 0;          // step of the next sequence forced to fail its conservation gate
    int cn_stage = 0;              // per-operator S2CN2 step: 1 after the evolution, 2 after the residual
    cudaGraphExec_t cgraph = nullptr;
    // the research wall variants of an S2CN2 context (ugks_s2_walls.cu)
    bool has_var = false;
    CnVariant V{};
    double* vmem = nullptr;
    unsigned* vflags = nullptr;    // [0] the predictor's last-CTA counter
    // S2CN2 adjoint (ugks_s2cn2_forward_checkpointed / ugks_s2cn2_backward / ugks_s2cn2_step_vjp)
    double* amem = nullptr;        // checkpoints (held from the checkpointed forward to the context's end)
    double* bmem = nullptr;        // segment slots, cotangent sets, adjoint work (reserved by the backward)
    double* rmem = nullptr;        // per-step records of one segment: the scratch each step's adjoint reads
    unsigned* aflags = nullptr;    // [0..2] halt, counter, accepted of the re-runs, [3] adjoint status
    int adj_capacity_ckpt = 0, adj_capacity_seg = 0, adj_capacity_rec = 0;
    cudaEvent_t adj_ev[4] = {nullptr, nullptr, nullptr, nullptr};   // the adjoint's fork / join points
    double* ckpt = nullptr;        // [ckpt][h | b | W | ledger]
    double* seg = nullptr;         // [slot][h | b | W | 6 targets | ledger]
    double* cot[2] = {nullptr, nullptr};   // [h | b | W | 6 targets] cotangent sets
    double* adj_seed = nullptr;    // [4]
    double* adj_ledger = nullptr;  // [16] the re-runs' ledger
    double* adj_report = nullptr;  // [kCnReport]
    AdjBuffers A{};
    int adj_nsteps = 0, adj_every = 0;   // the trajectory the checkpoints hold (0: none)
    int adj_last_recorded = 0;           // 1: the segment slots and records hold the trajectory's last segment
};

static int cuda_fail(cudaError_t e) {
    if (e == cudaSuccess) return UGKS_OK;
    std::fprintf(stderr, "ugks_b200: CUDA error %s\n", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? UGKS_ENOMEM : UGKS_ECUDA;
}

#define UGKS_CK(x)                                   \
    do {                                             \
        cudaError_t _e = (x);                        \
        if (_e != cudaSuccess) return cuda_fail(_e); \
    } while (0)

extern "C" const char* ugks_error_string(int code) {
    switch (code) {
        case UGKS_OK: return "ok";
        case UGKS_EINVAL: return "invalid argument";
        case UGKS_ECUDA: return "CUDA runtime error";
        case UGKS_ENUMERIC: return "device-side numerical gate failed";
        case UGKS_ETIMEOUT: return "bounded device wait expired";
        case UGKS_ENOMEM: return "out of device memory";
        case UGKS_EUNSUPPORTED: return "unsupported configuration";
        default: return "unknown";
    }
}

extern "C" int ugks_status_reference_code(unsigned st) {
    if (st & ST_GETPRIMARY) return 101;
    if (st & ST_TAU) return 104;
    if (st & ST_FACE_PROJECTION) return 446;
    if (st & ST_PROJECTION) return 444;
    if (st & ST_NONFINITE_FLUX) return 13;
    if (st & ST_NONFINITE_STATE) return 4;
    if (st & ST_STEP_REJECTED) return 203;
    if (st & ST_W1T_PREDICTOR) return 449;
    if (st & ST_W2R) return 456;
    if (st & ST_MOMENT_GATE) return 451;
    if (st & ST_ALPHA) return 433;
    if (st & ST_TIMEOUT) return 999;
    return 0;
}

// Read (and clear) the device status word; synchronises the stream.
static int collect_status(ugks_ctx* c) {
    unsigned st = 0;
    UGKS_CK(cudaMemcpyAsync(&st, c->dflags + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    if (st) UGKS_CK(cudaMemsetAsync(c->dflags + 1, 0, sizeof(unsigned), c->stream));
    c->last_status = st;
    if (st & ST_TIMEOUT) return UGKS_ETIMEOUT;
    return st ? UGKS_ENUMERIC : UGKS_OK;
}

// The research S2 wall variants a context accepts: the kinetic wall on both S2 methods (the implicit
// micro wall treatment does not depend on it, mod_ImplicitMicro.f90:701,777), W1T, W1D and W2R on S2CN2,
// in the combinations the reference's option checks admit (mod_ImportPara.f90:455-471, :527-528): W1T on
// the kinetic wall, W1D with W1T, W2R alone on the multiscale wall with ck = 1 and Pr = 1.
static int check_wall_variant(const ugks_params* p) {
    const int k = p->s2_kinetic_wall, t = p->s2_time_centered, d = p->s2_face_time, r = p->s2_shared_predictor;
    if ((k | t | d | r) & ~1) return UGKS_EINVAL;
    if (!(k | t | d | r)) return UGKS_OK;
    const bool ho_kinetic = p->method == UGKS_METHOD_HIGH_ORDER_IMPLICIT && !(t | d | r);
    if (p->method != UGKS_METHOD_S2CN2 && !ho_kinetic) return UGKS_EUNSUPPORTED;
    if (t && !k) return UGKS_EINVAL;
    if (d && !t) return UGKS_EINVAL;
    if (r && (k || t || d || p->ck != 1 || p->pr != 1.0)) return UGKS_EINVAL;
    return UGKS_OK;
}

extern "C" int ugks_ctx_create(const ugks_params* p, const double* u, const double* v, const double* w, int device,
                               ugks_ctx** out) {
    if (!p || !u || !v || !w || !out) return UGKS_EINVAL;
    if (int r = check_wall_variant(p)) return r;
    if (p->nx < 1 || p->ny < 3 || p->nvel < 1 || p->nvel > kMaxVel || !(p->dx > 0) || !(p->dy > 0) ||
        p->ck < 1)
        return UGKS_EINVAL;
    if (p->method != UGKS_METHOD_EXPLICIT && p->method != UGKS_METHOD_IMPLICIT_STEADY &&
        p->method != UGKS_METHOD_HIGH_ORDER_IMPLICIT && p->method != UGKS_METHOD_S2CN2)
        return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(device));
    ugks_ctx* c = new (std::nothrow) ugks_ctx();
    if (!c) return UGKS_ENOMEM;
    c->prm = *p;
    c->device = device;
    const int nx = p->nx, ny = p->ny, nv = p->nvel, nc = nx * ny;
    double umax = -INFINITY, vmax = -INFINITY;
    for (int k = 0; k < nv; ++k) { umax = std::fmax(umax, u[k]); vmax = std::fmax(vmax, v[k]); }
    c->P = make_lo_params(*p, umax, vmax);

    // buffer plan (doubles)
    const size_t S = (size_t)nc * nv, SY = (size_t)(ny + 1) * nx * nv;
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += (n + 31) / 32 * 32; return o; };
    const size_t o_u = take(nv), o_v = take(nv), o_w = take(nv);
    const size_t o_h = take(S), o_b = take(S), o_W = take((size_t)nc * 4);
    const size_t o_sxh = take(S), o_syh = take(S), o_sxb = take(S), o_syb = take(S);
    const size_t o_fxh = take(S), o_fxb = take(S), o_fxw = take((size_t)nc * 4);
    const size_t o_fyh = take(SY), o_fyb = take(SY), o_fyw = take((size_t)(ny + 1) * nx * 4);
    const size_t o_rw = take((size_t)nc * 4), o_rh = take(S), o_rb = take(S);
    const size_t o_eh = take(S), o_eb = take(S), o_ch = take(S), o_cb = take(S);
    const size_t o_dtl = take(nc), o_dt = take(2), o_cd = take((size_t)nc * kNDiag), o_dg = take(kNDiag);
    const size_t o_wa = take((size_t)2 * nx * 3);
    c->ndoubles = off;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&c->dmem, off * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c->dflags, 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->dmem, 0, off * sizeof(double), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->dflags, 0, 4 * sizeof(unsigned), c->stream);
    if (e != cudaSuccess) { ugks_ctx_destroy(c); return cuda_fail(e); }
    double* d = c->dmem;
    LoBuffers& B = c->B;
    B.u = d + o_u; B.v = d + o_v; B.w = d + o_w;
    B.h = d + o_h; B.b = d + o_b; B.W = d + o_W;
    B.sxh = d + o_sxh; B.syh = d + o_syh; B.sxb = d + o_sxb; B.syb = d + o_syb;
    B.fxh = d + o_fxh; B.fxb = d + o_fxb; B.fxw = d + o_fxw;
    B.fyh = d + o_fyh; B.fyb = d + o_fyb; B.fyw = d + o_fyw;
    B.res_w = d + o_rw; B.res_h = d + o_rh; B.res_b = d + o_rb;
    B.peq_h = d + o_eh; B.peq_b = d + o_eb; B.pcol_h = d + o_ch; B.pcol_b = d + o_cb;
    B.dtl = d + o_dtl; B.dt = d + o_dt; B.cell_diag = d + o_cd; B.diag = d + o_dg; B.wall_aero = d + o_wa;
    B.counter = c->dflags; B.status = c->dflags + 1;
    e = cudaMemcpyAsync(d + o_u, u, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + o_v, v, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + o_w, w, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    if (e == cudaSuccess && (p->method == UGKS_METHOD_IMPLICIT_STEADY || p->method == UGKS_METHOD_HIGH_ORDER_IMPLICIT)) {
        // ImplicitSteady work arrays (mod_ImplicitState.f90:110-132)
        ImParams& Q = c->Q;
        Q.nslab = p->nslab > 0 ? p->nslab : 1;
        Q.mass_rescale = p->mass_rescale;
        Q.macro_sweeps = p->macro_sweeps > 0 ? p->macro_sweeps : 2;
        Q.high_order = p->method == UGKS_METHOD_HIGH_ORDER_IMPLICIT ? 1 : 0;
        Q.ncfl = p->ncfl; Q.residual_tol = p->residual_tol; Q.moment_tol = p->moment_tol; Q.min_alpha = p->min_alpha;
        Q.wall_ux[0] = p->wall_ux[0]; Q.wall_ux[1] = p->wall_ux[1];
        if (ny % Q.nslab != 0 || (ny / Q.nslab) * nx > kMaxSlabCells) { ugks_ctx_destroy(c); return UGKS_EINVAL; }
        e = prepare_implicit(c->P, Q);
        size_t io = 0;
        auto itake = [&](size_t n) { size_t o = io; io += (n + 31) / 32 * 32; return o; };
        const size_t i_sh = itake(S), i_sb = itake(S), i_rw = itake((size_t)nc * 4), i_da = itake((size_t)nc * 4);
        const size_t i_db = itake((size_t)nc * 4), i_g = itake((size_t)nc * 4), i_fi = itake((size_t)nc * 16);
        const size_t i_fj = itake((size_t)nc * 16), i_wt = itake((size_t)nc * 4), i_tt = itake(nc);
        const size_t i_eh = itake(S), i_eb = itake(S), i_fh = itake(S), i_fb = itake(S), i_bh = itake(S), i_bb = itake(S);
        const size_t i_hu = itake((size_t)2 * nv), i_bu = itake((size_t)2 * nv), i_dr = itake((size_t)2 * nx);
        const size_t i_cell = itake((size_t)nc * kImCell), i_st = itake(IS_COUNT), i_rep = itake(kReport);
        // high order: the face cache (s2_rec_doubles) and the six volume targets
        const size_t i_rec = Q.high_order ? itake(s2_rec_doubles(nx, ny, nv)) : 0;
        size_t i_tg[6] = {0, 0, 0, 0, 0, 0};
        if (Q.high_order) for (int t = 0; t < 6; ++t) i_tg[t] = itake(S);
        const size_t i_scr = Q.high_order ? itake(s2_scratch_doubles(nx, ny, nv)) : 0;
        if (e == cudaSuccess && Q.high_order) e = prepare_s2();
        if (e == cudaSuccess) e = cudaMalloc(&c->imem, io * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&c->iflags, 6 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->imem, 0, io * sizeof(double), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->iflags, 0, 6 * sizeof(unsigned), c->stream);
        if (e == cudaSuccess) {
            double* m = c->imem;
            ImBuffers& I = c->I;
            I.stream_h = m + i_sh; I.stream_b = m + i_sb; I.rate_w = m + i_rw; I.dwA = m + i_da; I.dwB = m + i_db;
            I.pr_gamma = m + i_g; I.pr_foi = m + i_fi; I.pr_foj = m + i_fj; I.wt = m + i_wt; I.tau_t = m + i_tt;
            I.rhs_h = m + i_eh; I.rhs_b = m + i_eb; I.dFh = m + i_fh; I.dFb = m + i_fb; I.dBh = m + i_bh; I.dBb = m + i_bb;
            I.wall_hu = m + i_hu; I.wall_bu = m + i_bu; I.wall_drho = m + i_dr; I.cell = m + i_cell;
            I.state = m + i_st; I.report = m + i_rep;
            if (Q.high_order) {
                I.s2.rec = m + i_rec;
                I.s2.mh = m + i_tg[0]; I.s2.mb = m + i_tg[1]; I.s2.kxh = m + i_tg[2];
                I.s2.kxb = m + i_tg[3]; I.s2.kyh = m + i_tg[4]; I.s2.kyb = m + i_tg[5];
                s2_bind_scratch(I.s2, m + i_scr, nx, ny, nv);
            }
            I.mask = c->iflags; I.counter = c->iflags + 2; I.stopw = c->iflags + 3; I.prbar = c->iflags + 4;
        }
    }
    if (e == cudaSuccess && p->method == UGKS_METHOD_S2CN2) {
        // S2CN2: reconstruction cache, two target sets, the second state set, the stream state and the
        // CN right-hand side, per-cell diagnostics, ledger, report and raw wall fluxes
        size_t co = 0;
        auto ctake = [&](size_t n) { size_t o = co; co += (n + 31) / 32 * 32; return o; };
        const size_t c_rec = ctake(s2_rec_doubles(nx, ny, nv));
        size_t c_tg[2][6];
        for (int q = 0; q < 2; ++q) for (int t = 0; t < 6; ++t) c_tg[q][t] = ctake(S);
        const size_t c_h1 = ctake(S), c_b1 = ctake(S), c_W1 = ctake((size_t)nc * 4);
        const size_t c_ws = ctake((size_t)nc * 4), c_rh = ctake(S), c_rb = ctake(S);
        const size_t c_cell = ctake((size_t)nc * kCnCell), c_led = ctake(16), c_rep = ctake(kCnReport);
        const size_t c_wr = ctake((size_t)2 * nx * 4), c_scr = ctake(s2_scratch_doubles(nx, ny, nv));
        e = prepare_s2();
        if (e == cudaSuccess) e = cudaMalloc(&c->cmem, co * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&c->cflags, 4 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->cmem, 0, co * sizeof(double), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->cflags, 0, 4 * sizeof(unsigned), c->stream);
        if (e == cudaSuccess) {
            double* m = c->cmem;
            for (int q = 0; q < 2; ++q) {
                S2Buffers& T = c->T[q];
                T.rec = m + c_rec;
                T.mh = m + c_tg[q][0]; T.mb = m + c_tg[q][1]; T.kxh = m + c_tg[q][2];
                T.kxb = m + c_tg[q][3]; T.kyh = m + c_tg[q][4]; T.kyb = m + c_tg[q][5];
                T.wall_raw = m + c_wr;
                s2_bind_scratch(T, m + c_scr, nx, ny, nv);   // one evaluation at a time: shared by both sets
            }
            CnBuffers& C = c->C;
            C.ws = m + c_ws; C.rh = m + c_rh; C.rb = m + c_rb; C.cell = m + c_cell; C.ledger = m + c_led;
            C.report = m + c_rep; C.wall_raw = m + c_wr;
            C.halt = c->cflags; C.counter = c->cflags + 1; C.accepted = c->cflags + 2;
            c->Bs[0] = B;
            c->Bs[0].halt = C.halt;
            c->Bs[1] = c->Bs[0];
            c->Bs[1].h = m + c_h1; c->Bs[1].b = m + c_b1; c->Bs[1].W = m + c_W1;
        }
        const LoParams& P = c->P;
        if (e == cudaSuccess && (P.s2_kinetic || P.s2_midpoint || P.s2_shared)) {
            // the wall variant's buffers: coefficient outputs, the predictor's dt, face arrays, evaluation
            // set, stream state and the predicted state, the instantaneous wall node fluxes
            c->has_var = true;
            const size_t nfw = (size_t)nx * ny + (size_t)nx * (ny - 1) + 2 * (size_t)nx;
            size_t vo = 0;
            auto vtake = [&](size_t n) { size_t o = vo; vo += (n + 31) / 32 * 32; return o; };
            const bool coef = P.s2_face_time || P.s2_shared, pred = P.s2_midpoint || P.s2_shared;
            const size_t v_coef = coef ? vtake(nfw * 3 * 4 * nv) : 0;
            const size_t v_half = vtake(2), v_fxh = vtake(S), v_fxb = vtake(S), v_fxw = vtake((size_t)nc * 4);
            const size_t v_fyh = vtake(SY), v_fyb = vtake(SY), v_fyw = vtake((size_t)(ny + 1) * nx * 4);
            const size_t v_wa = vtake((size_t)2 * nx * 3);
            const size_t v_rec = pred ? vtake(s2_rec_doubles(nx, ny, nv)) : 0;
            size_t v_tg[6] = {0, 0, 0, 0, 0, 0};
            if (P.s2_midpoint) for (int t = 0; t < 6; ++t) v_tg[t] = vtake(S);
            const size_t v_scr = pred ? vtake(s2_scratch_doubles(nx, ny, nv)) : 0;
            const size_t v_ws = vtake((size_t)nc * 4), v_rh = vtake(S), v_rb = vtake(S), v_cell = vtake((size_t)nc * kCnCell);
            const size_t v_rep = vtake(kCnReport), v_h = vtake(S), v_b = vtake(S), v_W = vtake((size_t)nc * 4);
            const size_t v_inst = P.s2_shared ? vtake((size_t)2 * nx * 3 * 2 * nv) : 0;
            e = cudaMalloc(&c->vmem, vo * sizeof(double));
            if (e == cudaSuccess) e = cudaMalloc(&c->vflags, 4 * sizeof(unsigned));
            if (e == cudaSuccess) e = cudaMemsetAsync(c->vmem, 0, vo * sizeof(double), c->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(c->vflags, 0, 4 * sizeof(unsigned), c->stream);
            if (e == cudaSuccess) {
                double* m = c->vmem;
                CnVariant& V = c->V;
                if (coef) { c->T[0].coef = m + v_coef; c->T[1].coef = m + v_coef; }
                V.half = m + v_half;
                V.fxh = m + v_fxh; V.fxb = m + v_fxb; V.fxw = m + v_fxw;
                V.fyh = m + v_fyh; V.fyb = m + v_fyb; V.fyw = m + v_fyw; V.wall_aero = m + v_wa;
                if (pred) {
                    V.Sp.rec = m + v_rec;
                    s2_bind_scratch(V.Sp, m + v_scr, nx, ny, nv);
                }
                if (P.s2_midpoint) {
                    V.Sp.mh = m + v_tg[0]; V.Sp.mb = m + v_tg[1]; V.Sp.kxh = m + v_tg[2];
                    V.Sp.kxb = m + v_tg[3]; V.Sp.kyh = m + v_tg[4]; V.Sp.kyb = m + v_tg[5];
                }
                V.Cp.ws = m + v_ws; V.Cp.rh = m + v_rh; V.Cp.rb = m + v_rb; V.Cp.cell = m + v_cell;
                V.Cp.report = m + v_rep; V.Cp.ledger = nullptr; V.Cp.wall_raw = nullptr;
                V.Cp.halt = c->C.halt; V.Cp.counter = c->vflags; V.Cp.accepted = c->vflags + 1; V.Cp.predict = 1;
                V.h = m + v_h; V.b = m + v_b; V.W = m + v_W;
                V.inst = P.s2_shared ? m + v_inst : nullptr;
            }
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { ugks_ctx_destroy(c); return cuda_fail(e); }
    *out = c;
    return UGKS_OK;
}

extern "C" int ugks_ctx_destroy(ugks_ctx* c) {
    if (!c) return UGKS_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->igraph) cudaGraphExecDestroy(c->igraph);
    if (c->pgraph) cudaGraphExecDestroy(c->pgraph);
    if (c->iloop) cudaGraphExecDestroy(c->iloop);
    if (c->iloop_ctr) cudaFree(c->iloop_ctr);
    if (c->cgraph) cudaGraphExecDestroy(c->cgraph);
    if (c->amem) cudaFree(c->amem);
    if (c->bmem) cudaFree(c->bmem);
    if (c->rmem) cudaFree(c->rmem);
    for (int q = 0; q < 4; ++q) if (c->adj_ev[q]) cudaEventDestroy(c->adj_ev[q]);
    if (c->aflags) cudaFree(c->aflags);
    if (c->cmem) cudaFree(c->cmem);
    if (c->cflags) cudaFree(c->cflags);
    if (c->vmem) cudaFree(c->vmem);
    if (c->vflags) cudaFree(c->vflags);
    if (c->imem) cudaFree(c->imem);
    if (c->iflags) cudaFree(c->iflags);
    if (c->hstate) cudaFreeHost(c->hstate);
    if (c->icap.s) cudaStreamDestroy(c->icap.s);
    if (c->icap.s2) cudaStreamDestroy(c->icap.s2);
    if (c->icap.fork) cudaEventDestroy(c->icap.fork);
    if (c->icap.join) cudaEventDestroy(c->icap.join);
    for (int i = 0; i < 2; ++i) if (c->rb_ev[i]) cudaEventDestroy(c->rb_ev[i]);
    for (int i = 0; i < 5; ++i) if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (int i = 0; i <= kImStages; ++i) if (c->im_ev[i]) cudaEventDestroy(c->im_ev[i]);
    if (c->dmem) cudaFree(c->dmem);
    if (c->dflags) cudaFree(c->dflags);
    if (c->stream2) { cudaStreamSynchronize(c->stream2); cudaStreamDestroy(c->stream2); }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return UGKS_OK;
}

static int kernel_timestep(ugks_ctx* c) {
    UGKS_CK(launch_lo_timestep(c->P, c->B, c->stream));
    c->launches += 1;
    return UGKS_OK;
}

// Any call that changes the state, dt or the flux arrays outside the implicit step invalidates the
// cached accepted-state evaluation the next implicit step would otherwise reuse.
static int invalidate_eval(ugks_ctx* c) {
    if (c->imem) UGKS_CK(cudaMemsetAsync(c->I.state + IS_EVAL_VALID, 0, sizeof(double), c->stream));
    return UGKS_OK;
}

extern "C" int ugks_upload_state(ugks_ctx* c, const double* h, const double* b, const double* W) {
    if (!c || !h || !b || !W) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    UGKS_CK(cudaMemcpyAsync(c->B.h, h, S * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    UGKS_CK(cudaMemcpyAsync(c->B.b, b, S * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    UGKS_CK(cudaMemcpyAsync(c->B.W, W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    c->cn_ready = false;   // an S2CN2 context needs ugks_s2cn2_init for the new state
    c->cn_stage = 0;
    int r = kernel_timestep(c);
    if (r) return r;
    return collect_status(c);
}

extern "C" int ugks_download_state(ugks_ctx* c, double* h, double* b, double* W) {
    if (!c) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    if (h) UGKS_CK(cudaMemcpyAsync(h, c->B.h, S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (b) UGKS_CK(cudaMemcpyAsync(b, c->B.b, S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (W)
        UGKS_CK(cudaMemcpyAsync(W, c->B.W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

// h, b with the reference's LAP halo: host arrays [ny + 2 lap][nx + 2 lap][nvel], interior at (lap, lap).
// One strided copy per array; the halo of the host arrays is neither read nor written.
static cudaError_t copy_halo(double* dst, const double* src, const ugks_ctx* c, int lap, cudaMemcpyKind kind) {
    const size_t nv = (size_t)c->P.nvel, nx = (size_t)c->P.nx, ny = (size_t)c->P.ny;
    const size_t row = nx * nv * sizeof(double), hpitch = (nx + 2 * (size_t)lap) * nv * sizeof(double);
    const size_t hoff = ((size_t)lap * (nx + 2 * (size_t)lap) + (size_t)lap) * nv;
    if (kind == cudaMemcpyHostToDevice) return cudaMemcpy2DAsync(dst, row, src + hoff, hpitch, row, ny, kind, c->stream);
    return cudaMemcpy2DAsync(dst + hoff, hpitch, src, row, row, ny, kind, c->stream);
}

extern "C" int ugks_upload_state_halo(ugks_ctx* c, const double* h, const double* b, const double* W, int lap) {
    if (!c || !h || !b || !W || lap < 0) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    UGKS_CK(copy_halo(c->B.h, h, c, lap, cudaMemcpyHostToDevice));
    UGKS_CK(copy_halo(c->B.b, b, c, lap, cudaMemcpyHostToDevice));
    UGKS_CK(cudaMemcpyAsync(c->B.W, W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    c->cn_ready = false;
    c->cn_stage = 0;
    int r = kernel_timestep(c);
    if (r) return r;
    return collect_status(c);
}

extern "C" int ugks_download_state_halo(ugks_ctx* c, double* h, double* b, double* W, int lap) {
    if (!c || lap < 0) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (h) UGKS_CK(copy_halo(h, c->B.h, c, lap, cudaMemcpyDeviceToHost));
    if (b) UGKS_CK(copy_halo(b, c->B.b, c, lap, cudaMemcpyDeviceToHost));
    if (W)
        UGKS_CK(cudaMemcpyAsync(W, c->B.W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

extern "C" int ugks_init_freestream(ugks_ctx* c, double rho, double U, double V, double tnative) {
    if (!c || !(rho > 0) || !(tnative > 0)) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    UGKS_CK(launch_lo_init(c->P, c->B, rho, U, V, tnative, c->stream));
    c->launches += 1;
    if (c->imem && c->Q.high_order) {   // S2NativeInitializeState cold start: h, b := closure Maxwellian of W
        UGKS_CK(s2_enqueue(0, c->P, c->B, c->I.s2, c->stream, c->stream2, c->ev_fork, c->ev_join));
        c->launches += s2_enqueue_kernels(0);
    }
    if (c->cmem) {   // the same cold start, then the S2CN2 ledger and the targets of the state
        UGKS_CK(s2_enqueue(0, c->P, c->B, c->T[0], c->stream, c->stream2, c->ev_fork, c->ev_join));
        UGKS_CK(enqueue_s2cn2_prepare(c->P, c->Bs[0], c->T[0], c->C, c->stream, &c->launches));
        c->launches += s2_enqueue_kernels(0);
        c->cn_ready = true;
    }
    int r = kernel_timestep(c);
    if (r) return r;
    return collect_status(c);
}

extern "C" int ugks_timestep(ugks_ctx* c, double* dt_out) {
    if (!c) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    int r = kernel_timestep(c);
    if (r) return r;
    if (dt_out) UGKS_CK(cudaMemcpyAsync(dt_out, c->B.dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return collect_status(c);
}

// The S2 evolution of the current state (S2NativeEvolution, mod_S2NativeAdapter.f90:469-490): the
// high-order faces, walls and their macro fluxes, with the volume targets rebuilt (HighOrderImplicit
// always, S2CN2 when asked) or kept (S2CN2: the accepted state's targets from the last step or from
// ugks_s2cn2_init).  An S2CN2 evaluation starts a per-operator step: the halt flag, the accepted count
// and the rejection hook are armed as ugks_s2cn2_steps arms them for a sequence of one step.
static int s2_evolution(ugks_ctx* c, bool rebuild_targets) {
    if (c->cmem) {
        if (!c->cn_ready && !rebuild_targets) return UGKS_EINVAL;   // no targets: ugks_s2cn2_init first
        int r = collect_status(c);
        if (r) return r;
        UGKS_CK(cudaMemsetAsync(c->cflags, 0, 3 * sizeof(unsigned), c->stream));
        const double inject = (double)c->cn_reject_at;
        UGKS_CK(cudaMemcpyAsync(c->C.ledger + 8, &inject, sizeof inject, cudaMemcpyHostToDevice, c->stream));
        c->cn_reject_at = 0;
        const int which = rebuild_targets ? 1 : 2;
        UGKS_CK(s2_enqueue(which, c->P, c->Bs[0], c->T[0], c->stream, c->stream2, c->ev_fork, c->ev_join));
        c->launches += s2_enqueue_kernels(which);
        if (c->has_var) {   // the wall variant's part of S2NativeEvolution (mod_S2NativeAdapter.f90:491-540)
            UGKS_CK(enqueue_s2cn2_variant(c->P, c->Bs[0], c->T[0], c->V, c->stream, c->stream2, c->ev_fork,
                                          c->ev_join));
            c->launches += s2cn2_variant_kernels(c->P);
        }
        r = collect_status(c);
        c->cn_ready = c->cn_ready || (rebuild_targets && r == UGKS_OK);
        c->cn_stage = r == UGKS_OK ? 1 : 0;
        return r;
    }
    UGKS_CK(s2_enqueue(1, c->P, c->B, c->I.s2, c->stream, c->stream2, c->ev_fork, c->ev_join));
    c->launches += s2_enqueue_kernels(1);
    return collect_status(c);
}

static bool is_s2(const ugks_ctx* c) {
    return c->prm.method == UGKS_METHOD_S2CN2 || c->prm.method == UGKS_METHOD_HIGH_ORDER_IMPLICIT;
}

extern "C" int ugks_evolution(ugks_ctx* c) {
    if (!c) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    if (is_s2(c)) return s2_evolution(c, c->prm.method == UGKS_METHOD_HIGH_ORDER_IMPLICIT);
    UGKS_CK(launch_lo_slopes(c->P, c->B, c->stream));
    UGKS_CK(launch_lo_faces(c->P, c->B, c->stream));
    UGKS_CK(launch_lo_walls(c->P, c->B, c->stream));
    c->launches += 3;
    return collect_status(c);
}

extern "C" int ugks_evolution_s2(ugks_ctx* c, int rebuild_targets) {
    if (!c) return UGKS_EINVAL;
    if (!is_s2(c)) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    return s2_evolution(c, rebuild_targets != 0 || c->prm.method == UGKS_METHOD_HIGH_ORDER_IMPLICIT);
}

extern "C" int ugks_compute_residual(ugks_ctx* c, int with_collision) {
    if (!c) return UGKS_EINVAL;
    if (c->prm.method == UGKS_METHOD_HIGH_ORDER_IMPLICIT) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    if (c->cmem) {   // S2CN2: residual, stream state, S2 physical collision gate, CN right-hand side
        if (c->cn_stage != 1) return UGKS_EINVAL;
        UGKS_CK(enqueue_cn_stream(c->P, c->Bs[0], c->T[0], c->C, c->stream));
        c->launches += 1;
        const int r = collect_status(c);
        c->cn_stage = r == UGKS_OK ? 2 : 0;
        return r;
    }
    UGKS_CK(launch_lo_cells(c->P, c->B, 1, with_collision != 0, c->stream));
    c->launches += 1;
    return collect_status(c);
}

// S2NativeApplyUpdate (mod_S2NativeAdapter.f90:867-940) of a per-operator S2CN2 step: the targets of
// the stream state and the CN collision into state set 1, the gates and the acceptance; an accepted
// state (and its targets) is brought back to set 0.
static int s2cn2_apply(ugks_ctx* c) {
    if (c->cn_stage != 2) return UGKS_EINVAL;
    c->cn_stage = 0;
    UGKS_CK(enqueue_cn_apply(c->P, c->Bs[0], c->Bs[1], c->T[1], c->C, c->stream));
    c->launches += 1 + s2_enqueue_kernels(3);
    unsigned acc = 0;
    UGKS_CK(cudaMemcpyAsync(&acc, c->C.accepted, sizeof acc, cudaMemcpyDeviceToHost, c->stream));
    const int r = collect_status(c);
    if (acc == 1u) {
        const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].h, c->Bs[1].h, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].b, c->Bs[1].b, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].W, c->Bs[1].W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
        double* src[6] = {c->T[1].mh, c->T[1].mb, c->T[1].kxh, c->T[1].kxb, c->T[1].kyh, c->T[1].kyb};
        double* dst[6] = {c->T[0].mh, c->T[0].mb, c->T[0].kxh, c->T[0].kxb, c->T[0].kyh, c->T[0].kyb};
        for (int t = 0; t < 6; ++t)
            UGKS_CK(cudaMemcpyAsync(dst[t], src[t], S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaStreamSynchronize(c->stream));
    }
    return r;
}

static int read_step_outputs(ugks_ctx* c, double* dt_out, double* res_out) {
    double dg[kNDiag];
    if (res_out) UGKS_CK(cudaMemcpyAsync(dg, c->B.diag, sizeof dg, cudaMemcpyDeviceToHost, c->stream));
    int r = collect_status(c);
    if (res_out) finish_explicit_res(c->P.nx, c->P.ny, dg, res_out);
    (void)dt_out;
    return r;
}

extern "C" int ugks_apply_explicit_update(ugks_ctx* c, double* res_out) {
    if (!c) return UGKS_EINVAL;
    if (c->prm.method == UGKS_METHOD_HIGH_ORDER_IMPLICIT) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    if (c->cmem) return s2cn2_apply(c);
    UGKS_CK(launch_lo_cells(c->P, c->B, 2, false, c->stream));
    c->launches += 1;
    return read_step_outputs(c, nullptr, res_out);
}

// One Explicit step per iteration: slopes, then the interior faces on the main stream while the
// wall faces run on the side stream (they read only the slopes and the state), joined before the
// cell update.  The fork/join is recorded into the CUDA graph as two parallel branches.
static cudaError_t enqueue_explicit_steps(ugks_ctx* c, int n) {
    for (int s = 0; s < n; ++s) {
        cudaError_t e = launch_lo_slopes(c->P, c->B, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_fork, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream2, c->ev_fork, 0);
        if (e == cudaSuccess) e = launch_lo_walls(c->P, c->B, c->stream2);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_join, c->stream2);
        if (e == cudaSuccess) e = launch_lo_faces(c->P, c->B, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
        if (e == cudaSuccess) e = launch_lo_cells(c->P, c->B, 3, false, c->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static int build_graph(ugks_ctx* c, int steps) {
    if (c->graph && c->graph_steps == steps) return UGKS_OK;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    cudaGraph_t g;
    UGKS_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_explicit_steps(c, steps);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { if (e2 == cudaSuccess) cudaGraphDestroy(g); return cuda_fail(e); }
    UGKS_CK(e2);
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    UGKS_CK(e);
    c->graph_steps = steps;
    return UGKS_OK;
}

extern "C" int ugks_step_explicit(ugks_ctx* c, int nsteps, double* dt_out, double* res_out) {
    if (!c || nsteps < 0) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = invalidate_eval(c)) return r;
    if (nsteps == 0) return UGKS_OK;
    if (c->profile) {
        for (int s = 0; s < nsteps; ++s) {
            UGKS_CK(cudaEventRecord(c->ev[4], c->stream));
            UGKS_CK(launch_lo_slopes(c->P, c->B, c->stream));
            UGKS_CK(cudaEventRecord(c->ev[0], c->stream));
            UGKS_CK(launch_lo_faces(c->P, c->B, c->stream));
            UGKS_CK(cudaEventRecord(c->ev[1], c->stream));
            UGKS_CK(launch_lo_walls(c->P, c->B, c->stream));
            UGKS_CK(cudaEventRecord(c->ev[2], c->stream));
            UGKS_CK(launch_lo_cells(c->P, c->B, 3, false, c->stream));
            UGKS_CK(cudaEventRecord(c->ev[3], c->stream));
            UGKS_CK(cudaEventSynchronize(c->ev[3]));
            float a = 0.f, w = 0.f, b = 0.f, sl = 0.f;
            UGKS_CK(cudaEventElapsedTime(&sl, c->ev[4], c->ev[0]));
            UGKS_CK(cudaEventElapsedTime(&a, c->ev[0], c->ev[1]));
            UGKS_CK(cudaEventElapsedTime(&w, c->ev[1], c->ev[2]));
            UGKS_CK(cudaEventElapsedTime(&b, c->ev[2], c->ev[3]));
            c->t_slopes.total_ms += sl; c->t_slopes.launches += 1;
            c->t_faces.total_ms += a; c->t_faces.launches += 1;
            c->t_walls.total_ms += w; c->t_walls.launches += 1;
            c->t_cells.total_ms += b; c->t_cells.launches += 1;
        }
        c->launches += 4LL * nsteps;
    } else {
        const int G = 16;
        int full = nsteps / G, rem = nsteps % G;
        if (full > 0) {
            int r = build_graph(c, G);
            if (r) return r;
            for (int i = 0; i < full; ++i) UGKS_CK(cudaGraphLaunch(c->graph, c->stream));
        }
        UGKS_CK(enqueue_explicit_steps(c, rem));
        c->launches += 4LL * nsteps;
    }
    if (dt_out) UGKS_CK(cudaMemcpyAsync(dt_out, c->B.dt + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return read_step_outputs(c, dt_out, res_out);
}

extern "C" int ugks_macro_fields(ugks_ctx* c, double* out) {
    if (!c || !out) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->P.nx * c->P.ny * 10;
    double* d = nullptr;
    UGKS_CK(cudaMallocAsync(&d, n * sizeof(double), c->stream));
    cudaError_t e = launch_lo_macro_fields(c->P, c->B, d, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    UGKS_CK(e);
    c->launches += 1;
    return collect_status(c);
}

extern "C" int ugks_wall_aero(ugks_ctx* c, double* out) {
    if (!c || !out) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    UGKS_CK(cudaMemcpyAsync(out, c->B.wall_aero, (size_t)2 * c->P.nx * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

extern "C" int ugks_copy_array(ugks_ctx* c, const char* name, double* host, size_t n) {
    if (!c || !name || !host) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    const size_t nx = c->P.nx, ny = c->P.ny, nv = c->P.nvel, nc = nx * ny;
    const double* src = nullptr;
    size_t cnt = 0;
    const std::string s(name);
    if (s == "res_w") { src = c->B.res_w; cnt = nc * 4; }
    else if (s == "res_h") { src = c->B.res_h; cnt = nc * nv; }
    else if (s == "res_b") { src = c->B.res_b; cnt = nc * nv; }
    else if (s == "fxh") { src = c->B.fxh; cnt = nc * nv; }
    else if (s == "fxb") { src = c->B.fxb; cnt = nc * nv; }
    else if (s == "fxw") { src = c->B.fxw; cnt = nc * 4; }
    else if (s == "fyh") { src = c->B.fyh; cnt = (ny + 1) * nx * nv; }
    else if (s == "fyb") { src = c->B.fyb; cnt = (ny + 1) * nx * nv; }
    else if (s == "fyw") { src = c->B.fyw; cnt = (ny + 1) * nx * 4; }
    else if (s == "pcol_h") { src = c->B.pcol_h; cnt = nc * nv; }
    else if (s == "pcol_b") { src = c->B.pcol_b; cnt = nc * nv; }
    else if (s == "peq_h") { src = c->B.peq_h; cnt = nc * nv; }
    else if (s == "peq_b") { src = c->B.peq_b; cnt = nc * nv; }
    else if (s == "dt") { src = c->B.dt; cnt = 2; }
    else return UGKS_EINVAL;
    if (n < cnt) return UGKS_EINVAL;
    UGKS_CK(cudaMemcpyAsync(host, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

extern "C" unsigned ugks_last_status(const ugks_ctx* c) { return c ? c->last_status : 0u; }

extern "C" void* ugks_stream(ugks_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int ugks_synchronize(ugks_ctx* c) {
    if (!c) return UGKS_EINVAL;
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

extern "C" int ugks_profile_enable(ugks_ctx* c, int enable) {
    if (!c) return UGKS_EINVAL;
    c->profile = enable == 2 ? 2 : (enable != 0 ? 1 : 0);
    c->t_slopes = KernelTimer();
    c->t_faces = KernelTimer();
    c->t_walls = KernelTimer();
    c->t_cells = KernelTimer();
    for (int q = 0; q < kImStages; ++q) c->im_t[q] = KernelTimer();
    return UGKS_OK;
}

extern "C" int ugks_profile_read(ugks_ctx* c, const char* kernel, double* total_ms, long long* launches) {
    if (!c || !kernel) return UGKS_EINVAL;
    const KernelTimer* t = nullptr;
    if (!std::strcmp(kernel, "slopes")) t = &c->t_slopes;
    else if (!std::strcmp(kernel, "faces")) t = &c->t_faces;
    else if (!std::strcmp(kernel, "walls")) t = &c->t_walls;
    else if (!std::strcmp(kernel, "cells")) t = &c->t_cells;
    for (int q = 0; q < kImStages && !t; ++q)
        if (!std::strcmp(kernel, kImStageNames[q])) t = &c->im_t[q];
    if (!t) return UGKS_EINVAL;
    if (total_ms) *total_ms = t->total_ms;
    if (launches) *launches = t->launches;
    return UGKS_OK;
}

extern "C" long long ugks_launch_count(const ugks_ctx* c) { return c ? c->launches : 0; }

// ---------------------------------------------------------------------------------------------
// ImplicitSteady

extern "C" int ugks_implicit_init(ugks_ctx* c) {
    if (!c) return UGKS_EINVAL;
    if (!c->imem) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    UGKS_CK(launch_im_init(c->P, c->B, c->Q, c->I, c->stream));
    // + the first pseudo-step's pre-update S2 evaluation and residual (in graphs a conditional body)
    c->launches += 1 + (c->Q.high_order ? 1 + s2_enqueue_kernels(1) : 0);
    c->implicit_ready = true;
    return collect_status(c);
}

extern "C" int ugks_implicit_restore(ugks_ctx* c, double m0, double reference_h, double reference_b,
                                     int have_reference) {
    if (!c) return UGKS_EINVAL;
    if (!c->imem) return UGKS_EUNSUPPORTED;
    // ValidMass (finite, positive) for M0; the references must be finite when inherited
    if (!(std::isfinite(m0) && m0 > 0.0)) return UGKS_EINVAL;
    if (have_reference && !(std::isfinite(reference_h) && std::isfinite(reference_b))) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    UGKS_CK(launch_im_init(c->P, c->B, c->Q, c->I, c->stream));
    // + the first pseudo-step's pre-update S2 evaluation and residual (in graphs a conditional body)
    c->launches += 1 + (c->Q.high_order ? 1 + s2_enqueue_kernels(1) : 0);
    static_assert(IS_REF_H == IS_M0 + 1 && IS_REF_B == IS_M0 + 2 && IS_REF_INIT == IS_M0 + 3,
                  "M0 and the residual references are contiguous state words");
    const double v[4] = {m0, have_reference ? reference_h : 0.0, have_reference ? reference_b : 0.0,
                         have_reference ? 1.0 : 0.0};
    UGKS_CK(cudaMemcpyAsync(c->I.state + IS_M0, v, sizeof v, cudaMemcpyHostToDevice, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    c->implicit_ready = true;
    return collect_status(c);
}

static int build_implicit_graph(ugks_ctx* c, int steps) {
    if (c->igraph && c->igraph_steps == steps) return UGKS_OK;
    if (c->igraph) { cudaGraphExecDestroy(c->igraph); c->igraph = nullptr; }
    if (!c->icap.s) {
        UGKS_CK(cudaStreamCreateWithFlags(&c->icap.s, cudaStreamNonBlocking));
        UGKS_CK(cudaStreamCreateWithFlags(&c->icap.s2, cudaStreamNonBlocking));
        UGKS_CK(cudaEventCreateWithFlags(&c->icap.fork, cudaEventDisableTiming));
        UGKS_CK(cudaEventCreateWithFlags(&c->icap.join, cudaEventDisableTiming));
    }
    cudaGraph_t g;
    long long n = 0;
    UGKS_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < steps && e == cudaSuccess; ++s)
        // the S2 pre-update evaluation goes into a conditional body (its skipped kernels launch grids of
        // 16k CTAs); the second-order one keeps its launches, which return at entry more cheaply than the
        // conditional node costs
        e = enqueue_implicit_step(c->P, c->B, c->Q, c->I, c->stream, c->stream2, c->ev_fork, c->ev_join, &n, nullptr,
                                  c->Q.high_order ? &c->icap : nullptr);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { if (e2 == cudaSuccess) cudaGraphDestroy(g); return cuda_fail(e); }
    UGKS_CK(e2);
    e = cudaGraphInstantiate(&c->igraph, g, 0);
    cudaGraphDestroy(g);
    UGKS_CK(e);
    c->igraph_steps = steps;
    c->igraph_launches = n;
    return UGKS_OK;
}

// Batch budget of the device-driven pseudo-step loop, armed by the host before each loop launch.
__global__ void k_im_loop_arm(unsigned* ctr, unsigned batches) { *ctr = batches; }

// Last node of every loop iteration: spends one batch of the budget and continues only while budget
// remains, the sequence has not stopped and no kernel has raised a status bit (a failed gate of the
// evaluation kernels raises one without stopping the sequence; the call returns that failure, so
// nothing after the failing batch runs).  It sets the condition on every iteration, so the loop ends
// after at most the armed number of batches whatever the state holds.
__global__ void k_im_loop_cond(cudaGraphConditionalHandle h, unsigned* ctr, const double* state,
                               const unsigned* status) {
    const unsigned left = *ctr;
    const unsigned next = left > 0u ? left - 1u : 0u;
    *ctr = next;
    cudaGraphSetConditional(h, (next > 0u && state[IS_STOP] == 0.0 && *status == 0u) ? 1u : 0u);
}

// The device-driven form of the batch loop (second-order path): a graph whose WHILE node runs a body
// of `steps` pseudo-steps followed by k_im_loop_cond, so a whole call runs without the host.
static cudaError_t build_implicit_loop(ugks_ctx* c, int steps) {
    cudaError_t e = cudaSuccess;
    if (!c->iloop_ctr) e = cudaMalloc((void**)&c->iloop_ctr, sizeof(unsigned));
    cudaGraph_t g = nullptr;
    if (e == cudaSuccess) e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle h = 0;
    e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    long long n = 0;
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(c->stream, np.conditional.phGraph_out[0], nullptr, nullptr,
                                                           0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t eb = cudaSuccess;
        for (int s = 0; s < steps && eb == cudaSuccess; ++s)
            eb = enqueue_implicit_step(c->P, c->B, c->Q, c->I, c->stream, c->stream2, c->ev_fork, c->ev_join, &n,
                                       nullptr, nullptr);
        if (eb == cudaSuccess) {
            k_im_loop_cond<<<1, 1, 0, c->stream>>>(h, c->iloop_ctr, c->I.state, c->B.status);
            eb = cudaGetLastError();
        }
        cudaGraph_t body = nullptr;
        e = cudaStreamEndCapture(c->stream, &body);
        if (eb != cudaSuccess) e = eb;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&c->iloop, g, 0);
    cudaGraphDestroy(g);
    if (e == cudaSuccess) c->iloop_launches = n + 1;
    return e;
}

// Whether the device-driven loop runs this context's batches: the second-order path only (the S2 step
// holds a conditional node of its own), built on first use; if that build fails the host pipeline runs
// the batches instead.
static bool use_implicit_loop(ugks_ctx* c, int steps) {
    if (c->Q.high_order || c->iloop_unavailable) return false;
    if (c->iloop) return true;
    if (build_implicit_loop(c, steps) == cudaSuccess) return true;
    cudaGetLastError();
    c->iloop_unavailable = true;
    return false;
}

extern "C" int ugks_implicit_steps(ugks_ctx* c, int max_steps, int* steps_done, int* converged, double* report) {
    if (!c || max_steps < 0) return UGKS_EINVAL;
    if (!c->imem) return UGKS_EUNSUPPORTED;
    if (!c->implicit_ready) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    const int G = 8;
    double st[IS_COUNT];
    UGKS_CK(cudaMemcpyAsync(st, c->I.state, sizeof st, cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    const double start = st[IS_STEPS];
    int left = max_steps;
    if (left > 0 && st[IS_STOP] == 0.0) {   // the first pseudo-step's TimeStep (each later one's is taken by
        UGKS_CK(launch_lo_timestep(c->P, c->B, c->stream));   // the pseudo-step before it)
        c->launches += 1;
    }
    while (left > 0 && st[IS_STOP] == 0.0) {
        if (c->profile == 2 && left >= G) {
            // a batch graph with an external event node after every stage: the events keep the batch's last
            // pseudo-step, whose stages are timed as the graphs run them (no launch gaps of their own)
            for (int q = 0; q <= kImStages; ++q)
                if (!c->im_ev[q]) UGKS_CK(cudaEventCreate(&c->im_ev[q]));
            if (!c->pgraph) {
                cudaGraph_t g;
                long long n = 0;
                UGKS_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                cudaError_t e = cudaSuccess;
                for (int q = 0; q < G && e == cudaSuccess; ++q)
                    e = enqueue_implicit_step(c->P, c->B, c->Q, c->I, c->stream, c->stream2, c->ev_fork, c->ev_join, &n,
                                              c->im_ev, c->Q.high_order ? &c->icap : nullptr);
                cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
                if (e != cudaSuccess) { if (e2 == cudaSuccess) cudaGraphDestroy(g); return cuda_fail(e); }
                UGKS_CK(e2);
                e = cudaGraphInstantiate(&c->pgraph, g, 0);
                cudaGraphDestroy(g);
                UGKS_CK(e);
                c->igraph_launches = n;
            }
            UGKS_CK(cudaGraphLaunch(c->pgraph, c->stream));
            UGKS_CK(cudaMemcpyAsync(st, c->I.state, sizeof st, cudaMemcpyDeviceToHost, c->stream));
            UGKS_CK(cudaStreamSynchronize(c->stream));
            for (int q = 0; q < kImStages; ++q) {
                float ms = 0.f;
                UGKS_CK(cudaEventElapsedTime(&ms, c->im_ev[q], c->im_ev[q + 1]));
                c->im_t[q].total_ms += ms;
                c->im_t[q].launches += 1;
            }
            c->launches += c->igraph_launches;
            left -= G;
            if (int r = collect_status(c)) return r;
            continue;
        }
        if (c->profile) {   // un-graphed, one step at a time, with an event after every stage
            for (int q = 0; q <= kImStages; ++q)
                if (!c->im_ev[q]) UGKS_CK(cudaEventCreate(&c->im_ev[q]));
            long long n = 0;
            UGKS_CK(enqueue_implicit_step(c->P, c->B, c->Q, c->I, c->stream, c->stream2, c->ev_fork, c->ev_join, &n,
                                          c->im_ev));
            UGKS_CK(cudaEventSynchronize(c->im_ev[kImStages]));
            for (int q = 0; q < kImStages; ++q) {
                float ms = 0.f;
                UGKS_CK(cudaEventElapsedTime(&ms, c->im_ev[q], c->im_ev[q + 1]));
                c->im_t[q].total_ms += ms;
                c->im_t[q].launches += 1;
            }
            c->launches += n;
            left -= 1;
        } else if (left >= G && use_implicit_loop(c, G)) {
            // The device runs the batches: one launch of the WHILE-node graph, bounded by the batch budget
            // (after a stop, the rest of the stopping batch's kernels return at entry)
            const unsigned nb = (unsigned)(left / G);
            unsigned rest = 0;
            k_im_loop_arm<<<1, 1, 0, c->stream>>>(c->iloop_ctr, nb);
            UGKS_CK(cudaGetLastError());
            UGKS_CK(cudaGraphLaunch(c->iloop, c->stream));
            UGKS_CK(cudaMemcpyAsync(&rest, c->iloop_ctr, sizeof rest, cudaMemcpyDeviceToHost, c->stream));
            UGKS_CK(cudaMemcpyAsync(st, c->I.state, sizeof st, cudaMemcpyDeviceToHost, c->stream));
            UGKS_CK(cudaStreamSynchronize(c->stream));
            const long long ran = (long long)nb - (long long)rest;
            if (ran < 1 || ran > (long long)nb) return cuda_fail(cudaErrorUnknown);   // the loop body did not run
            c->launches += 1 + c->iloop_launches * ran;
            left -= G * (int)ran;
            continue;
        } else if (left >= G) {
            // Batches of up to 2 graphs, each followed by a copy of the state into a pinned slot.  The
            // next batch is queued before the host waits for the previous batch's copy, so the device
            // never idles on the host between batches.  After a stop the queued steps' kernels return
            // at entry, so the state and the counts stay those of the stopping step.
            int r = build_implicit_graph(c, G);
            if (r) return r;
            if (!c->hstate) {
                UGKS_CK(cudaMallocHost((void**)&c->hstate, 2 * IS_COUNT * sizeof(double)));
                for (int i = 0; i < 2; ++i) UGKS_CK(cudaEventCreateWithFlags(&c->rb_ev[i], cudaEventDisableTiming));
            }
            auto queue_batch = [&](int slot) -> cudaError_t {
                const int ng = left / G < 2 ? left / G : 2;
                for (int q = 0; q < ng; ++q) {
                    const cudaError_t e = cudaGraphLaunch(c->igraph, c->stream);
                    if (e != cudaSuccess) return e;
                }
                c->launches += c->igraph_launches * ng;
                left -= G * ng;
                const cudaError_t e = cudaMemcpyAsync(c->hstate + slot * IS_COUNT, c->I.state, IS_COUNT * sizeof(double),
                                                      cudaMemcpyDeviceToHost, c->stream);
                return e != cudaSuccess ? e : cudaEventRecord(c->rb_ev[slot], c->stream);
            };
            int cur = 0;
            UGKS_CK(queue_batch(cur));
            for (;;) {
                const int prev = cur;
                cur = left >= G ? 1 - prev : -1;
                if (cur >= 0) UGKS_CK(queue_batch(cur));
                UGKS_CK(cudaEventSynchronize(c->rb_ev[prev]));
                std::memcpy(st, c->hstate + prev * IS_COUNT, sizeof st);
                if (st[IS_STOP] != 0.0 || cur < 0) break;
            }
            if (cur >= 0) {   // a batch queued past the stop: let it drain, then read the final state
                UGKS_CK(cudaMemcpyAsync(st, c->I.state, sizeof st, cudaMemcpyDeviceToHost, c->stream));
                UGKS_CK(cudaStreamSynchronize(c->stream));
            }
            continue;
        } else {
            long long n = 0;
            for (int s = 0; s < left; ++s)
                UGKS_CK(enqueue_implicit_step(c->P, c->B, c->Q, c->I, c->stream, c->stream2, c->ev_fork,
                                              c->ev_join, &n, nullptr));
            c->launches += n;
            left = 0;
        }
        UGKS_CK(cudaMemcpyAsync(st, c->I.state, sizeof st, cudaMemcpyDeviceToHost, c->stream));
        UGKS_CK(cudaStreamSynchronize(c->stream));
    }
    if (steps_done) *steps_done = (int)(st[IS_STEPS] - start);
    if (converged) *converged = st[IS_CONVERGED] != 0.0 ? 1 : 0;
    if (report) UGKS_CK(cudaMemcpyAsync(report, c->I.report, kReport * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return collect_status(c);
}

extern "C" int ugks_implicit_state(ugks_ctx* c, double* state, double* report) {
    if (!c || !c->imem) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (state) UGKS_CK(cudaMemcpyAsync(state, c->I.state, kStatePublic * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (report) UGKS_CK(cudaMemcpyAsync(report, c->I.report, kReport * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

// ---------------------------------------------------------------------------------------------
// S2CN2

extern "C" int ugks_s2cn2_init(ugks_ctx* c) {
    if (!c) return UGKS_EINVAL;
    if (!c->cmem) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    UGKS_CK(enqueue_s2cn2_prepare(c->P, c->Bs[0], c->T[0], c->C, c->stream, &c->launches));
    const int r = collect_status(c);
    c->cn_ready = r == UGKS_OK;
    c->cn_stage = 0;
    return r;
}

extern "C" int ugks_s2cn2_test_reject(ugks_ctx* c, int step) {
    if (!c || step < 0) return UGKS_EINVAL;
    if (!c->cmem) return UGKS_EUNSUPPORTED;
    c->cn_reject_at = step;
    return UGKS_OK;
}

extern "C" int ugks_s2cn2_report(ugks_ctx* c, double* report) {
    if (!c || !report) return UGKS_EINVAL;
    if (!c->cmem) return UGKS_EUNSUPPORTED;
    UGKS_CK(cudaSetDevice(c->device));
    UGKS_CK(cudaMemcpyAsync(report, c->C.report, kCnReport * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

// one step of a ugks_s2cn2_steps sequence: its dt is the one the previous step's k_cn_collide took from the
// state it accepted (the sequence's first from the k_lo_timestep ugks_s2cn2_steps launches first)
static cudaError_t enqueue_cn_step(ugks_ctx* c, int from) {
    return enqueue_s2cn2_step(c->P, c->Bs[from], c->T[from], c->Bs[1 - from], c->T[1 - from], c->C, c->stream,
                              c->stream2, c->ev_fork, c->ev_join, nullptr, c->has_var ? &c->V : nullptr, false);
}

// a pair of steps, set 0 -> set 1 -> set 0, captured once and replayed
static int build_cn_graph(ugks_ctx* c) {
    if (c->cgraph) return UGKS_OK;
    cudaGraph_t g;
    UGKS_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_cn_step(c, 0);
    if (e == cudaSuccess) e = enqueue_cn_step(c, 1);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) { if (e2 == cudaSuccess) cudaGraphDestroy(g); return cuda_fail(e); }
    UGKS_CK(e2);
    e = cudaGraphInstantiate(&c->cgraph, g, 0);
    cudaGraphDestroy(g);
    UGKS_CK(e);
    return UGKS_OK;
}

extern "C" int ugks_s2cn2_steps(ugks_ctx* c, int nsteps, int* steps_done, double* report) {
    if (!c || nsteps < 0) return UGKS_EINVAL;
    if (!c->cmem) return UGKS_EUNSUPPORTED;
    if (!c->cn_ready) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (steps_done) *steps_done = 0;
    c->cn_stage = 0;
    // a new sequence: clear the halt flag and the accepted count, and any stale status
    int r = collect_status(c);
    if (r) return r;
    UGKS_CK(cudaMemsetAsync(c->cflags, 0, 3 * sizeof(unsigned), c->stream));
    const double inject = (double)c->cn_reject_at;
    UGKS_CK(cudaMemcpyAsync(c->C.ledger + 8, &inject, sizeof inject, cudaMemcpyHostToDevice, c->stream));
    c->cn_reject_at = 0;
    if (nsteps > 0) {   // the first step's TimeStep
        UGKS_CK(launch_lo_timestep(c->P, c->Bs[0], c->stream));
        c->launches += 1;
    }
    const int pairs = nsteps / 2;
    if (pairs > 0) {
        r = build_cn_graph(c);
        if (r) return r;
        for (int q = 0; q < pairs; ++q) UGKS_CK(cudaGraphLaunch(c->cgraph, c->stream));
    }
    if (nsteps % 2) UGKS_CK(enqueue_cn_step(c, 0));
    c->launches += (long long)(kCnStepKernels - 1 + (c->has_var ? s2cn2_variant_kernels(c->P) : 0)) * nsteps;
    unsigned acc = 0;
    UGKS_CK(cudaMemcpyAsync(&acc, c->C.accepted, sizeof acc, cudaMemcpyDeviceToHost, c->stream));
    if (report) UGKS_CK(cudaMemcpyAsync(report, c->C.report, kCnReport * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    r = collect_status(c);
    if (acc % 2) {   // the last accepted state is in set 1: bring it (and its targets) back to set 0
        const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].h, c->Bs[1].h, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].b, c->Bs[1].b, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaMemcpyAsync(c->Bs[0].W, c->Bs[1].W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
        double* src[6] = {c->T[1].mh, c->T[1].mb, c->T[1].kxh, c->T[1].kxb, c->T[1].kyh, c->T[1].kyb};
        double* dst[6] = {c->T[0].mh, c->T[0].mb, c->T[0].kxh, c->T[0].kxb, c->T[0].kyh, c->T[0].kyb};
        for (int t = 0; t < 6; ++t)
            UGKS_CK(cudaMemcpyAsync(dst[t], src[t], S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        UGKS_CK(cudaStreamSynchronize(c->stream));
    }
    if (steps_done) *steps_done = (int)acc;
    return r;
}

// ---------------------------------------------------------------------------------------------
// S2CN2 adjoint: checkpointed forward, reverse sweep with recompute, one-step VJP

namespace {

size_t rnd32(size_t n) { return (n + 31) / 32 * 32; }

struct SlotView {
    double *h, *b, *W, *T[6], *ledger;
};

size_t state_doubles(const ugks_ctx* c) {
    const size_t nc = (size_t)c->P.nx * c->P.ny, S = nc * c->P.nvel;
    return 2 * rnd32(S) + rnd32(nc * 4);
}
size_t ckpt_doubles(const ugks_ctx* c) { return state_doubles(c) + 32; }
size_t seg_doubles(const ugks_ctx* c) {
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    return state_doubles(c) + 6 * rnd32(S) + 32;
}
size_t cot_doubles(const ugks_ctx* c) {
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    return state_doubles(c) + 6 * rnd32(S);
}

// h, b, W (and, with targets, the six targets) of a block laid out as state_doubles + 6 targets
SlotView view_of(const ugks_ctx* c, double* base, bool targets, bool ledger) {
    const size_t nc = (size_t)c->P.nx * c->P.ny, S = nc * c->P.nvel;
    SlotView v{};
    v.h = base; base += rnd32(S);
    v.b = base; base += rnd32(S);
    v.W = base; base += rnd32(nc * 4);
    for (int t = 0; t < 6; ++t) {
        v.T[t] = targets ? base : nullptr;
        if (targets) base += rnd32(S);
    }
    v.ledger = ledger ? base : nullptr;
    return v;
}
SlotView ckpt_view(const ugks_ctx* c, int q) { return view_of(c, c->ckpt + (size_t)q * ckpt_doubles(c), false, true); }
SlotView seg_view(const ugks_ctx* c, int m) { return view_of(c, c->seg + (size_t)m * seg_doubles(c), true, true); }
SlotView cot_view(const ugks_ctx* c, int i) { return view_of(c, c->cot[i], true, false); }

// A step's record: what its adjoint reads of the step's evaluation and update -- the face cache, the
// first layer, the face-node scalars, the wall-node macro fluxes, the stream state's volume-node states
// and scalars, the CN right-hand side and the stream state.  The segment recompute writes step m's
// into record m, so the reverse sweep needs no second run of the step.
size_t record_doubles(const ugks_ctx* c) {
    const size_t nx = c->P.nx, ny = c->P.ny, nv = c->P.nvel, nc = nx * ny, S = nc * nv;
    const size_t nf = nc + nx * (ny - 1), nfw = nf + 2 * nx;
    return rnd32(s2_rec_doubles((int)nx, (int)ny, (int)nv)) + rnd32(nc * 22 * nv) + rnd32(nf * 3 * kS2FScal) + rnd32(nfw * 3 * 4) +
           rnd32(nc * 9 * 4) + rnd32(nc * 9 * kS2TScal) + 2 * rnd32(S) + rnd32(nc * 4);
}
// T with its evaluation scratch in record m (node and mac, which the adjoint does not read, stay shared)
S2Buffers with_record(const ugks_ctx* c, S2Buffers T, int m) {
    const size_t nx = c->P.nx, ny = c->P.ny, nv = c->P.nvel, nc = nx * ny;
    const size_t nf = nc + nx * (ny - 1), nfw = nf + 2 * nx;
    double* r = c->rmem + (size_t)m * record_doubles(c);
    T.rec = r; r += rnd32(s2_rec_doubles((int)nx, (int)ny, (int)nv));
    T.l1 = r; r += rnd32(nc * 22 * nv);
    T.fscal = r; r += rnd32(nf * 3 * kS2FScal);
    T.nodew = r; r += rnd32(nfw * 3 * 4);
    T.wq = r; r += rnd32(nc * 9 * 4);
    T.tscal = r;
    return T;
}
// the step buffers (rerun_cn) with the stream state and the CN right-hand side in record m
CnBuffers record_cn(const ugks_ctx* c, CnBuffers C, int m) {
    const size_t nx = c->P.nx, ny = c->P.ny, nv = c->P.nvel, nc = nx * ny, S = nc * nv;
    const size_t nf = nc + nx * (ny - 1), nfw = nf + 2 * nx;
    double* r = c->rmem + (size_t)m * record_doubles(c) + rnd32(s2_rec_doubles((int)nx, (int)ny, (int)nv)) + rnd32(nc * 22 * nv) +
                rnd32(nf * 3 * kS2FScal) + rnd32(nfw * 3 * 4) + rnd32(nc * 9 * 4) + rnd32(nc * 9 * kS2TScal);
    C.rh = r; r += rnd32(S);
    C.rb = r; r += rnd32(S);
    C.ws = r;
    return C;
}

// the state set of a slot: the context's set 0 with the slot's arrays and the re-runs' halt flag
LoBuffers slot_lo(const ugks_ctx* c, const SlotView& v) {
    LoBuffers B = c->Bs[0];
    B.h = v.h; B.b = v.b; B.W = v.W;
    B.halt = c->aflags;
    return B;
}
S2Buffers slot_targets(const ugks_ctx* c, const SlotView& v) {
    S2Buffers T = c->T[0];
    T.mh = v.T[0]; T.mb = v.T[1]; T.kxh = v.T[2]; T.kxb = v.T[3]; T.kyh = v.T[4]; T.kyb = v.T[5];
    return T;
}
// the re-runs' step buffers: the shared stream state and right-hand side, a ledger, report and flags of
// their own, so that a re-run never touches the accepted sequence's ledger
CnBuffers rerun_cn(const ugks_ctx* c) {
    CnBuffers C = c->C;
    C.ledger = c->adj_ledger;
    C.report = c->adj_report;
    C.halt = c->aflags;
    C.counter = c->aflags + 1;
    C.accepted = c->aflags + 2;
    return C;
}
AdjBuffers adj_bind(const ugks_ctx* c, int out, const double* seed) {
    AdjBuffers A = c->A;
    const SlotView o = cot_view(c, out), in = cot_view(c, 1 - out);
    A.gho = o.h; A.gbo = o.b; A.gWo = o.W;
    A.ghi = in.h; A.gbi = in.b; A.gWi = in.W;
    for (int t = 0; t < 6; ++t) { A.gTo[t] = o.T[t]; A.gTi[t] = in.T[t]; }
    A.seed = seed;
    return A;
}

cudaError_t copy_state(const ugks_ctx* c, const SlotView& dst, const double* h, const double* b, const double* W) {
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    cudaError_t e = cudaMemcpyAsync(dst.h, h, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.b, b, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst.W, W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    return e;
}
// a ledger copy without the test-rejection hook (slot 8)
cudaError_t copy_ledger(const ugks_ctx* c, double* dst, const double* src) {
    cudaError_t e = cudaMemcpyAsync(dst, src, 8 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dst + 8, 0, sizeof(double), c->stream);
    return e;
}

// one step of the S2CN2 sequence from (Bin, Tin) into (Bout, Tout) with the ledger `ledger`, as
// enqueue_s2cn2_step, on the re-runs' buffers
cudaError_t rerun_step(ugks_ctx* c, const LoBuffers& Bin, const S2Buffers& Tin, const LoBuffers& Bout,
                       const S2Buffers& Tout, const double* ledger) {
    cudaError_t e = cudaMemsetAsync(c->aflags, 0, 3 * sizeof(unsigned), c->stream);
    if (e == cudaSuccess) e = copy_ledger(c, c->adj_ledger, ledger);
    if (e == cudaSuccess)
        e = enqueue_s2cn2_step(c->P, Bin, Tin, Bout, Tout, rerun_cn(c), c->stream, c->stream2, c->ev_fork, c->ev_join,
                               &c->launches);
    return e;
}

// the same with the step buffers C (a record's stream state and right-hand side)
cudaError_t rerun_step_into(ugks_ctx* c, const LoBuffers& Bin, const S2Buffers& Tin, const LoBuffers& Bout,
                            const S2Buffers& Tout, const double* ledger, const CnBuffers& C) {
    cudaError_t e = cudaMemsetAsync(c->aflags, 0, 3 * sizeof(unsigned), c->stream);
    if (e == cudaSuccess) e = copy_ledger(c, c->adj_ledger, ledger);
    if (e == cudaSuccess)
        e = enqueue_s2cn2_step(c->P, Bin, Tin, Bout, Tout, C, c->stream, c->stream2, c->ev_fork, c->ev_join, &c->launches);
    return e;
}

// the checkpoints of a trajectory (the checkpointed forward); kept until the next reservation or the
// context's end
int adj_reserve_ckpt(ugks_ctx* c, int nckpt) {
    if (c->amem && c->adj_capacity_ckpt >= nckpt) return UGKS_OK;
    if (c->amem) { cudaFree(c->amem); c->amem = nullptr; c->adj_capacity_ckpt = 0; }
    UGKS_CK(cudaMalloc(&c->amem, (size_t)nckpt * ckpt_doubles(c) * sizeof(double)));
    c->ckpt = c->amem;
    c->adj_capacity_ckpt = nckpt;
    return UGKS_OK;
}

// the reverse sweep's work: nseg segment slots, the two cotangent sets and the adjoint's arrays
int adj_reserve_bwd(ugks_ctx* c, int nseg) {
    for (int q = 0; q < 4; ++q)
        if (!c->adj_ev[q]) UGKS_CK(cudaEventCreateWithFlags(&c->adj_ev[q], cudaEventDisableTiming));
    if (!c->aflags) {
        UGKS_CK(cudaMalloc(&c->aflags, 4 * sizeof(unsigned)));
        UGKS_CK(cudaMemsetAsync(c->aflags, 0, 4 * sizeof(unsigned), c->stream));
    }
    if (c->bmem && c->adj_capacity_seg >= nseg) return UGKS_OK;
    if (c->bmem) { cudaFree(c->bmem); c->bmem = nullptr; c->adj_capacity_seg = 0; }
    const size_t nx = c->P.nx, ny = c->P.ny, nv = c->P.nvel;
    const size_t work = rnd32(adj_work_doubles((int)nx, (int)ny, (int)nv));
    const size_t tot = (size_t)nseg * seg_doubles(c) + 2 * cot_doubles(c) + work + 3 * 32;
    UGKS_CK(prepare_s2_adjoint());
    UGKS_CK(cudaMalloc(&c->bmem, tot * sizeof(double)));
    UGKS_CK(cudaMemsetAsync(c->bmem, 0, tot * sizeof(double), c->stream));
    double* m = c->bmem;
    c->seg = m; m += (size_t)nseg * seg_doubles(c);
    c->cot[0] = m; m += cot_doubles(c);
    c->cot[1] = m; m += cot_doubles(c);
    adj_bind_work(c->A, m, (int)nx, (int)ny, (int)nv);
    m += work;
    c->adj_seed = m; m += 32;
    c->adj_ledger = m; m += 32;
    c->adj_report = m;
    c->A.status = c->aflags + 3;
    c->adj_capacity_seg = nseg;
    return UGKS_OK;
}

// records for a segment of `len` steps, when they fit in 3/4 of the free device memory; otherwise none
// (the reverse sweep then runs every step a second time for its scratch).  Kept with the context.
bool adj_reserve_records(ugks_ctx* c, int len) {
    if (c->rmem && c->adj_capacity_rec >= len) return true;
    if (c->rmem) { cudaFree(c->rmem); c->rmem = nullptr; c->adj_capacity_rec = 0; }
    size_t freeb = 0, totb = 0;
    if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) { cudaGetLastError(); return false; }
    const size_t need = (size_t)len * record_doubles(c) * sizeof(double);
    if (need > freeb / 4 * 3) return false;
    if (cudaMalloc(&c->rmem, need) != cudaSuccess) { cudaGetLastError(); c->rmem = nullptr; return false; }
    c->adj_capacity_rec = len;
    return true;
}

// cotangent sets, parameter cotangents and the seed for a new reverse sweep
int adj_clear(ugks_ctx* c, const double* seed) {
    UGKS_CK(cudaMemsetAsync(c->cot[0], 0, 2 * cot_doubles(c) * sizeof(double), c->stream));
    UGKS_CK(cudaMemsetAsync(c->A.gpar, 0, GP_COUNT * sizeof(double), c->stream));
    UGKS_CK(cudaMemsetAsync(c->aflags + 3, 0, sizeof(unsigned), c->stream));
    double sd[4] = {0.0, 0.0, 0.0, 0.0};
    if (seed) for (int q = 0; q < 4; ++q) sd[q] = seed[q];
    UGKS_CK(cudaMemcpyAsync(c->adj_seed, sd, sizeof sd, cudaMemcpyHostToDevice, c->stream));
    return UGKS_OK;
}

// synchronise; the forward status word and the adjoint's own
int adj_status(ugks_ctx* c) {
    unsigned ast = 0;
    UGKS_CK(cudaMemcpyAsync(&ast, c->aflags + 3, sizeof ast, cudaMemcpyDeviceToHost, c->stream));
    const int r = collect_status(c);
    if (r) return r;
    c->last_status = ast;
    return ast ? UGKS_ENUMERIC : UGKS_OK;
}

int adj_outputs(ugks_ctx* c, double* out) {
    if (!out) return UGKS_OK;
    const int nx = c->P.nx;
    double* a = new (std::nothrow) double[(size_t)2 * nx * 3];
    if (!a) return UGKS_ENOMEM;
    cudaError_t e = cudaMemcpyAsync(a, c->B.wall_aero, (size_t)2 * nx * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess)
        for (int w = 0; w < 2; ++w) {
            double sh = 0.0, ht = 0.0;
            for (int i = 0; i < nx; ++i) { sh += a[((size_t)w * nx + i) * 3 + 1]; ht += a[((size_t)w * nx + i) * 3 + 2]; }
            out[2 * w] = sh / nx;
            out[2 * w + 1] = ht / nx;
        }
    delete[] a;
    return cuda_fail(e);
}

int adj_download(ugks_ctx* c, const SlotView& v, double* gh, double* gb, double* gW, double* grad) {
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    if (gh) UGKS_CK(cudaMemcpyAsync(gh, v.h, S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (gb) UGKS_CK(cudaMemcpyAsync(gb, v.b, S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (gW) UGKS_CK(cudaMemcpyAsync(gW, v.W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
    if (grad) UGKS_CK(cudaMemcpyAsync(grad, c->A.gpar, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    return UGKS_OK;
}

}  // namespace

// The trajectory's last segment, run step by step: step m reads segment slot m and writes slot m + 1
// (the proposal) and its adjoint record m, on the accepted sequence's ledger, report and flags, with the
// kernels and the order of ugks_s2cn2_steps (so the states are its states bit for bit).  The last
// accepted state then goes back to set 0 with its targets.  Returns the accepted count in *done.
int forward_recorded(ugks_ctx* c, int len, int* done) {
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    *done = 0;
    c->cn_stage = 0;
    if (int r = collect_status(c)) return r;
    UGKS_CK(cudaMemsetAsync(c->cflags, 0, 3 * sizeof(unsigned), c->stream));
    const double inject = (double)c->cn_reject_at;
    UGKS_CK(cudaMemcpyAsync(c->C.ledger + 8, &inject, sizeof inject, cudaMemcpyHostToDevice, c->stream));
    c->cn_reject_at = 0;
    const SlotView s0 = seg_view(c, 0);
    UGKS_CK(copy_state(c, s0, c->Bs[0].h, c->Bs[0].b, c->Bs[0].W));
    const double* kept[6] = {c->T[0].mh, c->T[0].mb, c->T[0].kxh, c->T[0].kxb, c->T[0].kyh, c->T[0].kyb};
    for (int t = 0; t < 6; ++t)
        UGKS_CK(cudaMemcpyAsync(s0.T[t], kept[t], S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    for (int m = 0; m < len; ++m) {
        const SlotView a = seg_view(c, m), b = seg_view(c, m + 1);
        LoBuffers Ba = slot_lo(c, a), Bb = slot_lo(c, b);
        Ba.halt = Bb.halt = c->C.halt;
        UGKS_CK(enqueue_s2cn2_step(c->P, Ba, with_record(c, slot_targets(c, a), m), Bb,
                                   with_record(c, slot_targets(c, b), m), record_cn(c, c->C, m), c->stream, c->stream2,
                                   c->ev_fork, c->ev_join, &c->launches));
    }
    unsigned acc = 0;
    UGKS_CK(cudaMemcpyAsync(&acc, c->C.accepted, sizeof acc, cudaMemcpyDeviceToHost, c->stream));
    const int r = collect_status(c);
    const SlotView e = seg_view(c, (int)acc);   // the last accepted state
    UGKS_CK(cudaMemcpyAsync(c->Bs[0].h, e.h, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    UGKS_CK(cudaMemcpyAsync(c->Bs[0].b, e.b, S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    UGKS_CK(cudaMemcpyAsync(c->Bs[0].W, e.W, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
    double* dst[6] = {c->T[0].mh, c->T[0].mb, c->T[0].kxh, c->T[0].kxb, c->T[0].kyh, c->T[0].kyb};
    for (int t = 0; t < 6; ++t)
        UGKS_CK(cudaMemcpyAsync(dst[t], e.T[t], S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    UGKS_CK(cudaStreamSynchronize(c->stream));
    *done = (int)acc;
    return r;
}

extern "C" int ugks_s2cn2_forward_checkpointed(ugks_ctx* c, int nsteps, int every, double* outputs) {
    if (!c || nsteps < 1 || every < 1) return UGKS_EINVAL;
    if (!c->cmem || c->has_var) return UGKS_EUNSUPPORTED;   // the adjoint transposes the delivered walls only
    if (!c->cn_ready) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    const int nckpt = (nsteps + every - 1) / every, seglen = every < nsteps ? every : nsteps;
    if (int r = adj_reserve_ckpt(c, nckpt)) return r;
    c->adj_nsteps = 0;
    c->adj_last_recorded = 0;
    // the last segment leaves its states and records for the reverse sweep, which then starts without
    // recomputing it, when the records fit
    if (int r = adj_reserve_bwd(c, seglen + 1)) return r;
    const bool record_last = adj_reserve_records(c, seglen);
    for (int q = 0; q < nckpt; ++q) {
        const SlotView v = ckpt_view(c, q);
        UGKS_CK(copy_state(c, v, c->Bs[0].h, c->Bs[0].b, c->Bs[0].W));
        UGKS_CK(copy_ledger(c, v.ledger, c->C.ledger));
        const int n = (q + 1) * every <= nsteps ? every : nsteps - q * every;
        int done = 0;
        const int r = record_last && q == nckpt - 1 ? forward_recorded(c, n, &done) : ugks_s2cn2_steps(c, n, &done, nullptr);
        if (r) return r;
        if (done != n) return UGKS_ENUMERIC;
    }
    c->adj_last_recorded = record_last ? 1 : 0;
    c->adj_nsteps = nsteps;
    c->adj_every = every;
    return adj_outputs(c, outputs);
}

extern "C" int ugks_s2cn2_backward(ugks_ctx* c, const double* seed, double* grad, double* gh0, double* gb0,
                                   double* gW0) {
    if (!c || !seed) return UGKS_EINVAL;
    if (!c->cmem || c->has_var) return UGKS_EUNSUPPORTED;   // the adjoint transposes the delivered walls only
    if (c->adj_nsteps < 1) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = collect_status(c)) return r;
    const int nsteps = c->adj_nsteps, every = c->adj_every, nckpt = (nsteps + every - 1) / every;
    const int seglen = every < nsteps ? every : nsteps;
    if (int r = adj_reserve_bwd(c, seglen + 1)) return r;
    const bool records = adj_reserve_records(c, seglen);
    if (int r = adj_clear(c, seed)) return r;
    const CnBuffers Cr = rerun_cn(c);
    int cur = 0;
    for (int q = nckpt - 1; q >= 0; --q) {
        const int n0 = q * every, len = n0 + every <= nsteps ? every : nsteps - n0;
        const SlotView ck = ckpt_view(c, q), s0 = seg_view(c, 0);
        // the last segment's states and records may still be those of the forward
        const bool held = records && q == nckpt - 1 && c->adj_last_recorded;
        if (!held) {
            UGKS_CK(copy_state(c, s0, ck.h, ck.b, ck.W));
            UGKS_CK(copy_ledger(c, s0.ledger, ck.ledger));
            UGKS_CK(s2_enqueue(3, c->P, slot_lo(c, s0), slot_targets(c, s0), c->stream, c->stream, nullptr, nullptr));
            c->launches += s2_enqueue_kernels(3);
        }
        if (records) {
            // the segment recomputed once from its checkpoint, each step leaving its record; then the
            // adjoints in reverse order from the records
            for (int m = 0; m < len && !held; ++m) {
                const SlotView a = seg_view(c, m), b = seg_view(c, m + 1);
                UGKS_CK(rerun_step_into(c, slot_lo(c, a), with_record(c, slot_targets(c, a), m), slot_lo(c, b),
                                        with_record(c, slot_targets(c, b), m), a.ledger, record_cn(c, Cr, m)));
                UGKS_CK(copy_ledger(c, b.ledger, c->adj_ledger));
            }
            for (int m = len - 1; m >= 0; --m) {
                const SlotView a = seg_view(c, m), b = seg_view(c, m + 1);
                const bool last = q == nckpt - 1 && m == len - 1;
                const AdjBuffers A = adj_bind(c, cur, last ? c->adj_seed : nullptr);
                const S2Buffers Sm = with_record(c, slot_targets(c, a), m);
                UGKS_CK(enqueue_s2cn2_adjoint(c->P, slot_lo(c, a), Sm, Sm, with_record(c, slot_targets(c, b), m),
                                              record_cn(c, Cr, m), A, c->stream, c->stream2, c->adj_ev));
                c->launches += kAdjStepKernels;
                cur = 1 - cur;
            }
        } else {
            for (int m = 0; m + 1 < len; ++m) {   // the segment's states, recomputed from its checkpoint
                const SlotView a = seg_view(c, m), b = seg_view(c, m + 1);
                UGKS_CK(rerun_step(c, slot_lo(c, a), slot_targets(c, a), slot_lo(c, b), slot_targets(c, b), a.ledger));
                UGKS_CK(copy_ledger(c, b.ledger, c->adj_ledger));
            }
            for (int m = len - 1; m >= 0; --m) {   // reverse: re-run the step for its scratch, then its adjoint
                const SlotView a = seg_view(c, m);
                const LoBuffers Ba = slot_lo(c, a);
                const S2Buffers Ta = slot_targets(c, a);
                LoBuffers Bs1 = c->Bs[1];
                Bs1.halt = c->aflags;
                UGKS_CK(rerun_step(c, Ba, Ta, Bs1, c->T[1], a.ledger));
                const bool last = q == nckpt - 1 && m == len - 1;
                const AdjBuffers A = adj_bind(c, cur, last ? c->adj_seed : nullptr);
                UGKS_CK(enqueue_s2cn2_adjoint(c->P, Ba, c->T[0], Ta, c->T[1], Cr, A, c->stream, c->stream2, c->adj_ev));
                c->launches += kAdjStepKernels;
                cur = 1 - cur;
            }
        }
        if (int r = adj_status(c)) return r;
    }
    if (nckpt > 1) c->adj_last_recorded = 0;   // the slots and records now hold the first segment
    const SlotView g = cot_view(c, cur);
    if (gh0 || gb0 || gW0) {   // x_0's targets depend on its W: their cotangent goes to W
        const SlotView s0 = seg_view(c, 0);
        UGKS_CK(s2_enqueue(3, c->P, slot_lo(c, s0), c->T[1], c->stream, c->stream, nullptr, nullptr));
        const AdjBuffers A = adj_bind(c, 1 - cur, nullptr);
        UGKS_CK(enqueue_targets_adjoint(c->P, slot_lo(c, s0), c->T[0], g.T, g.W, A, c->stream));
        c->launches += s2_enqueue_kernels(3) + 2;
        if (int r = adj_status(c)) return r;
    }
    return adj_download(c, g, gh0, gb0, gW0, grad);
}

extern "C" int ugks_s2cn2_step_vjp(ugks_ctx* c, const double* gh, const double* gb, const double* gW, const double* seed,
                                   double* gh_in, double* gb_in, double* gW_in, double* grad) {
    if (!c) return UGKS_EINVAL;
    if (!c->cmem || c->has_var) return UGKS_EUNSUPPORTED;   // the adjoint transposes the delivered walls only
    if (!c->cn_ready) return UGKS_EINVAL;
    UGKS_CK(cudaSetDevice(c->device));
    if (int r = adj_reserve_bwd(c, c->adj_capacity_seg > 0 ? c->adj_capacity_seg : 1)) return r;
    if (int r = collect_status(c)) return r;
    if (int r = adj_clear(c, seed)) return r;
    const size_t S = (size_t)c->P.nx * c->P.ny * c->P.nvel;
    const SlotView o = cot_view(c, 0), in = cot_view(c, 1);
    if (gh) UGKS_CK(cudaMemcpyAsync(o.h, gh, S * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (gb) UGKS_CK(cudaMemcpyAsync(o.b, gb, S * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (gW) UGKS_CK(cudaMemcpyAsync(o.W, gW, (size_t)c->P.nx * c->P.ny * 4 * sizeof(double), cudaMemcpyHostToDevice,
                                    c->stream));
    LoBuffers B0 = c->Bs[0];
    B0.halt = c->aflags;
    LoBuffers Bs1 = c->Bs[1];
    Bs1.halt = c->aflags;
    UGKS_CK(rerun_step(c, B0, c->T[0], Bs1, c->T[1], c->C.ledger));
    const AdjBuffers A = adj_bind(c, 0, c->adj_seed);
    UGKS_CK(enqueue_s2cn2_adjoint(c->P, B0, c->T[0], c->T[0], c->T[1], rerun_cn(c), A, c->stream, c->stream2, c->adj_ev));
    UGKS_CK(s2_enqueue(3, c->P, B0, c->T[1], c->stream, c->stream, nullptr, nullptr));   // W's targets, for their adjoint
    UGKS_CK(enqueue_targets_adjoint(c->P, B0, c->T[0], in.T, in.W, A, c->stream));
    c->launches += kAdjStepKernels + s2_enqueue_kernels(3) + 2;
    if (int r = adj_status(c)) return r;
    return adj_download(c, in, gh_in, gb_in, gW_in, grad);
}
