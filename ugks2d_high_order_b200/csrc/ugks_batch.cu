// ugks_batch.cu -- many independent S2CN2 Couette instances of uneven grid and velocity-set sizes
// advanced together: one CUDA graph launch per pair of steps for all instances.
//
// Memory: each instance owns only what persists between steps -- its velocity table, the two state
// sets (h, b, W), the two target sets, dt, the conservation ledger, the report and its flags (about
// 16 doubles per cell-velocity).  Everything a step writes and reads back within the step (the
// reconstruction cache, the first layer, node fluxes, face arrays, the stream state and CN right-hand
// side) lives in K scratch slots, each sized for the largest instance.  Instances are assigned to
// slots by a largest-first greedy on cells x velocities; a slot runs its instances one after another
// on its own stream (and side stream), and the K slots run concurrently.  The graph captures two
// steps (set 0 -> 1 -> 0) of every instance as K parallel branches.  ugks_batch_tune times the
// candidate slot counts on the live batch and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/ugks_b200.h"
#include "ugks_s2cn2.cuh"

namespace ugks {
cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_init(const LoParams& P, const LoBuffers& B, double rho, double U, double V, double tn,
                           cudaStream_t s);
}
using namespace ugks;

namespace {

struct Inst {
    LoParams P{};
    LoBuffers B[2] = {};   // state sets 0 and 1 (the scratch pointers are the slot's)
    S2Buffers T[2] = {};
    CnBuffers C{};
    double* mem = nullptr;     // persistent arrays
    unsigned* flags = nullptr; // [0] counter [1] status [2] halt [3] accepted  (inside the batch's flag array)
    size_t S = 0;              // cells x velocities
    int slot = 0;
    double tinf = 2.0;
};

struct BSlot {
    cudaStream_t s = nullptr, s2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, done = nullptr;
};

size_t rnd(size_t n) { return (n + 31) / 32 * 32; }

// doubles of per-step scratch one instance needs
size_t scratch_doubles(int nx, int ny, int nv) {
    const size_t nc = (size_t)nx * ny, S = nc * nv, SY = (size_t)(ny + 1) * nx * nv;
    return rnd(s2_rec_doubles(nx, ny, nv)) + rnd(s2_scratch_doubles(nx, ny, nv)) + 2 * rnd(S) + 2 * rnd(SY) + rnd(nc * 4) +
           rnd((size_t)(ny + 1) * nx * 4) + rnd(nc) + rnd(nc * kNDiag) + rnd(kNDiag) + rnd(nc * 4) + 2 * rnd(S) +
           rnd(nc * kCnCell) + rnd((size_t)2 * nx * 4);
}

}  // namespace

struct ugks_batch {
    int device = 0, n = 0, max_slots = 0, slots = 0;
    std::vector<Inst> inst;
    std::vector<BSlot> slot;
    double* scratch = nullptr;   // max_slots x per_slot
    size_t per_slot = 0;
    unsigned* flags = nullptr;   // [n][4]
    cudaStream_t origin = nullptr;
    cudaEvent_t ev0 = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
};

static int bfail(cudaError_t e) {
    if (e == cudaSuccess) return UGKS_OK;
    std::fprintf(stderr, "ugks_b200 batch: CUDA error %s\n", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? UGKS_ENOMEM : UGKS_ECUDA;
}
#define BCK(x)                                   \
    do {                                         \
        cudaError_t _e = (x);                    \
        if (_e != cudaSuccess) return bfail(_e); \
    } while (0)

// point an instance's per-step arrays into its slot's scratch
static void bind_scratch(ugks_batch* b, Inst& I) {
    const LoParams& P = I.P;
    const int nx = P.nx, ny = P.ny, nv = P.nvel;
    const size_t nc = (size_t)nx * ny, S = I.S, SY = (size_t)(ny + 1) * nx * nv;
    double* m = b->scratch + (size_t)I.slot * b->per_slot;
    auto take = [&](size_t k) { double* p = m; m += rnd(k); return p; };
    double* rec = take(s2_rec_doubles(nx, ny, nv));
    double* s2s = take(s2_scratch_doubles(nx, ny, nv));
    double *fxh = take(S), *fxb = take(S), *fyh = take(SY), *fyb = take(SY), *fxw = take(nc * 4);
    double* fyw = take((size_t)(ny + 1) * nx * 4);
    double *dtl = take(nc), *cd = take(nc * kNDiag), *dg = take(kNDiag);
    double *ws = take(nc * 4), *rh = take(S), *rb = take(S), *cell = take(nc * kCnCell);
    double* wraw = take((size_t)2 * nx * 4);
    for (int q = 0; q < 2; ++q) {
        LoBuffers& B = I.B[q];
        B.fxh = fxh; B.fxb = fxb; B.fyh = fyh; B.fyb = fyb; B.fxw = fxw; B.fyw = fyw;
        B.dtl = dtl; B.cell_diag = cd; B.diag = dg;
        S2Buffers& T = I.T[q];
        T.rec = rec;
        T.wall_raw = wraw;
        T.concurrent = 1;
        s2_bind_scratch(T, s2s, nx, ny, nv);
    }
    I.C.ws = ws; I.C.rh = rh; I.C.rb = rb; I.C.cell = cell; I.C.wall_raw = wraw;
}

// largest-first greedy assignment of instances to k slots
static void assign(ugks_batch* b, int k) {
    std::vector<int> order(b->n);
    for (int i = 0; i < b->n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->inst[x].S > b->inst[y].S; });
    std::vector<double> load(k, 0.0);
    for (int i : order) {
        const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->inst[i].slot = s;
        load[s] += (double)b->inst[i].S;
    }
    b->slots = k;
    for (auto& I : b->inst) bind_scratch(b, I);
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
}

extern "C" int ugks_batch_create(int n, const ugks_instance_desc* desc, int device, int max_streams, ugks_batch** out) {
    if (n < 1 || !desc || !out || max_streams < 1) return UGKS_EINVAL;
    for (int i = 0; i < n; ++i) {
        const ugks_params* p = &desc[i].params;
        if (!desc[i].u || !desc[i].v || !desc[i].w || p->method != UGKS_METHOD_S2CN2 || p->nx < 1 || p->ny < 6 ||
            p->nvel < 1 || p->nvel > kMaxVel || !(p->dx > 0) || !(p->dy > 0) || p->ck < 1)
            return UGKS_EINVAL;
        // the research wall variants run on single contexts only
        if (p->s2_kinetic_wall || p->s2_time_centered || p->s2_face_time || p->s2_shared_predictor)
            return UGKS_EUNSUPPORTED;
    }
    BCK(cudaSetDevice(device));
    ugks_batch* b = new (std::nothrow) ugks_batch();
    if (!b) return UGKS_ENOMEM;
    b->device = device;
    b->n = n;
    b->max_slots = std::min(max_streams, n);
    b->inst.resize(n);
    b->slot.resize(b->max_slots);
    cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev0, cudaEventDisableTiming);
    for (auto& s : b->slot) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.s2, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = prepare_s2();
    size_t per_slot = 0;
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        const ugks_params* p = &desc[i].params;
        Inst& I = b->inst[i];
        LoParams& P = I.P;
        double umax = -INFINITY, vmax = -INFINITY;
        for (int k = 0; k < p->nvel; ++k) { umax = std::fmax(umax, desc[i].u[k]); vmax = std::fmax(vmax, desc[i].v[k]); }
        P = make_lo_params(*p, umax, vmax);
        const int nx = p->nx, ny = p->ny, nv = p->nvel;
        const size_t nc = (size_t)nx * ny, S = nc * nv;
        I.S = S;
        per_slot = std::max(per_slot, scratch_doubles(nx, ny, nv));
        // persistent: u v w | h b W (x2) | targets (x2) | dt | ledger | report | wall_aero
        const size_t tot = 3 * rnd(nv) + 2 * (2 * rnd(S) + rnd(nc * 4)) + 12 * rnd(S) + rnd(2) + rnd(16) +
                           rnd(kCnReport) + rnd((size_t)2 * nx * 3);
        e = cudaMalloc(&I.mem, tot * sizeof(double));
        if (e == cudaSuccess) e = cudaMemsetAsync(I.mem, 0, tot * sizeof(double), b->origin);
        if (e != cudaSuccess) break;
        double* m = I.mem;
        auto take = [&](size_t k) { double* q = m; m += rnd(k); return q; };
        double *u = take(nv), *v = take(nv), *w = take(nv);
        e = cudaMemcpyAsync(u, desc[i].u, nv * sizeof(double), cudaMemcpyHostToDevice, b->origin);
        if (e == cudaSuccess) e = cudaMemcpyAsync(v, desc[i].v, nv * sizeof(double), cudaMemcpyHostToDevice, b->origin);
        if (e == cudaSuccess) e = cudaMemcpyAsync(w, desc[i].w, nv * sizeof(double), cudaMemcpyHostToDevice, b->origin);
        for (int q = 0; q < 2; ++q) {
            LoBuffers& B = I.B[q];
            B.u = u; B.v = v; B.w = w;
            B.h = take(S); B.b = take(S); B.W = take(nc * 4);
        }
        for (int q = 0; q < 2; ++q) {
            S2Buffers& T = I.T[q];
            T.mh = take(S); T.mb = take(S); T.kxh = take(S); T.kxb = take(S); T.kyh = take(S); T.kyb = take(S);
        }
        double* dt = take(2);
        I.C.ledger = take(16);
        I.C.report = take(kCnReport);
        double* wa = take((size_t)2 * nx * 3);
        for (int q = 0; q < 2; ++q) { I.B[q].dt = dt; I.B[q].wall_aero = wa; }
    }
    if (e == cudaSuccess) {
        b->per_slot = per_slot;
        e = cudaMalloc(&b->scratch, per_slot * b->max_slots * sizeof(double));
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->flags, (size_t)n * 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->flags, 0, (size_t)n * 4 * sizeof(unsigned), b->origin);
    if (e == cudaSuccess) {
        for (int i = 0; i < n; ++i) {
            Inst& I = b->inst[i];
            I.flags = b->flags + 4 * i;
            I.C.counter = I.flags + 0;
            I.C.halt = I.flags + 2;
            I.C.accepted = I.flags + 3;
            for (int q = 0; q < 2; ++q) {
                I.B[q].counter = I.flags + 0;
                I.B[q].status = I.flags + 1;
                I.B[q].halt = I.C.halt;
                I.B[q].eval = nullptr;
            }
        }
        assign(b, b->max_slots);
        e = cudaStreamSynchronize(b->origin);
    }
    if (e != cudaSuccess) { ugks_batch_destroy(b); return bfail(e); }
    *out = b;
    return UGKS_OK;
}

extern "C" int ugks_batch_destroy(ugks_batch* b) {
    if (!b) return UGKS_OK;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& I : b->inst) if (I.mem) cudaFree(I.mem);
    if (b->scratch) cudaFree(b->scratch);
    if (b->flags) cudaFree(b->flags);
    for (auto& s : b->slot) {
        if (s.s) cudaStreamDestroy(s.s);
        if (s.s2) cudaStreamDestroy(s.s2);
        if (s.fork) cudaEventDestroy(s.fork);
        if (s.join) cudaEventDestroy(s.join);
        if (s.done) cudaEventDestroy(s.done);
    }
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->origin) cudaStreamDestroy(b->origin);
    delete b;
    return UGKS_OK;
}

// the steps of every instance from state set p0 (1 or 2 steps), K branches forked from `origin`
static cudaError_t enqueue_all(ugks_batch* b, int nsteps) {
    cudaError_t e = cudaEventRecord(b->ev0, b->origin);
    for (int s = 0; s < b->slots && e == cudaSuccess; ++s) e = cudaStreamWaitEvent(b->slot[s].s, b->ev0, 0);
    for (int st = 0; st < nsteps && e == cudaSuccess; ++st) {
        const int p = st & 1;
        for (int i = 0; i < b->n && e == cudaSuccess; ++i) {
            Inst& I = b->inst[i];
            const BSlot& S = b->slot[I.slot];
            // dt from the previous step's collide (the run's first step: the k_lo_timestep ugks_batch_run launches)
            e = enqueue_s2cn2_step(I.P, I.B[p], I.T[p], I.B[1 - p], I.T[1 - p], I.C, S.s, S.s2, S.fork, S.join, nullptr,
                                   nullptr, false);
        }
    }
    for (int s = 0; s < b->slots && e == cudaSuccess; ++s) {
        e = cudaEventRecord(b->slot[s].done, b->slot[s].s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->origin, b->slot[s].done, 0);
    }
    return e;
}

static int build_graph(ugks_batch* b) {
    if (b->graph) return UGKS_OK;
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_all(b, 2);
    cudaError_t e2 = cudaStreamEndCapture(b->origin, &g);
    if (e != cudaSuccess) { if (e2 == cudaSuccess) cudaGraphDestroy(g); return bfail(e); }
    BCK(e2);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    BCK(e);
    return UGKS_OK;
}

extern "C" int ugks_batch_init_freestream(ugks_batch* b, double rho, double U, double V, double tnative) {
    if (!b || !(rho > 0) || !(tnative > 0)) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    BCK(cudaMemsetAsync(b->flags, 0, (size_t)b->n * 4 * sizeof(unsigned), b->origin));
    BCK(cudaStreamSynchronize(b->origin));
    for (auto& I : b->inst) {
        const BSlot& S = b->slot[I.slot];
        BCK(launch_lo_init(I.P, I.B[0], rho, U, V, tnative, S.s));
        BCK(s2_enqueue(0, I.P, I.B[0], I.T[0], S.s, S.s2, S.fork, S.join));
        BCK(enqueue_s2cn2_prepare(I.P, I.B[0], I.T[0], I.C, S.s, nullptr));
        b->launches += 1 + s2_enqueue_kernels(0) + 1 + s2_enqueue_kernels(3);   // init, cold start, prepare
    }
    BCK(cudaDeviceSynchronize());
    std::vector<unsigned> f((size_t)b->n * 4);
    BCK(cudaMemcpy(f.data(), b->flags, f.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->n; ++i)
        if (f[4 * i + 1]) return UGKS_ENUMERIC;
    return UGKS_OK;
}

// copy an instance's accepted state and targets from set 1 back to set 0
static cudaError_t copy_back(const Inst& I, cudaStream_t s) {
    const size_t S = I.S, nc = (size_t)I.P.nx * I.P.ny;
    cudaError_t e = cudaMemcpyAsync(I.B[0].h, I.B[1].h, S * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(I.B[0].b, I.B[1].b, S * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(I.B[0].W, I.B[1].W, nc * 4 * sizeof(double), cudaMemcpyDeviceToDevice, s);
    double* src[6] = {I.T[1].mh, I.T[1].mb, I.T[1].kxh, I.T[1].kxb, I.T[1].kyh, I.T[1].kyb};
    double* dst[6] = {I.T[0].mh, I.T[0].mb, I.T[0].kxh, I.T[0].kxb, I.T[0].kyh, I.T[0].kyb};
    for (int t = 0; t < 6 && e == cudaSuccess; ++t)
        e = cudaMemcpyAsync(dst[t], src[t], S * sizeof(double), cudaMemcpyDeviceToDevice, s);
    return e;
}

extern "C" int ugks_batch_run(ugks_batch* b, int nsteps, int* steps_done, unsigned* status) {
    if (!b || nsteps < 0) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    // a new sequence for every instance: clear counters, status, halt and accepted counts
    BCK(cudaMemsetAsync(b->flags, 0, (size_t)b->n * 4 * sizeof(unsigned), b->origin));
    if (nsteps > 0)   // every instance's first TimeStep; each later step's dt is taken by the step before it
        for (auto& I : b->inst) BCK(launch_lo_timestep(I.P, I.B[0], b->origin));
    const int pairs = nsteps / 2;
    if (pairs > 0) {
        int r = build_graph(b);
        if (r) return r;
        for (int q = 0; q < pairs; ++q) BCK(cudaGraphLaunch(b->graph, b->origin));
    }
    if (nsteps % 2) BCK(enqueue_all(b, 1));
    b->launches += ((long long)(kCnStepKernels - 1) * nsteps + (nsteps > 0 ? 1 : 0)) * b->n;
    std::vector<unsigned> f((size_t)b->n * 4);
    BCK(cudaMemcpyAsync(f.data(), b->flags, f.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, b->origin));
    BCK(cudaStreamSynchronize(b->origin));
    bool bad = false;
    for (int i = 0; i < b->n; ++i) {
        const unsigned acc = f[4 * i + 3];
        if (steps_done) steps_done[i] = (int)acc;
        if (status) status[i] = f[4 * i + 1];
        bad = bad || f[4 * i + 1] != 0u;
        if (acc % 2) BCK(copy_back(b->inst[i], b->origin));
    }
    BCK(cudaStreamSynchronize(b->origin));
    return bad ? UGKS_ENUMERIC : UGKS_OK;
}

extern "C" int ugks_batch_tune(ugks_batch* b, int steps, int* chosen, double* ms_per_step) {
    if (!b || steps < 2) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    cudaEvent_t t0, t1;
    BCK(cudaEventCreate(&t0));
    BCK(cudaEventCreate(&t1));
    int best = b->slots;
    float best_ms = INFINITY;
    std::vector<int> cand;
    for (int k = 1; k < b->max_slots; k *= 2) cand.push_back(k);
    cand.push_back(b->max_slots);
    for (int k : cand) {
        assign(b, k);
        int r = ugks_batch_run(b, 2, nullptr, nullptr);   // graph build and warm-up
        if (r) { cudaEventDestroy(t0); cudaEventDestroy(t1); return r; }
        BCK(cudaEventRecord(t0, b->origin));
        r = ugks_batch_run(b, steps, nullptr, nullptr);
        if (r) { cudaEventDestroy(t0); cudaEventDestroy(t1); return r; }
        BCK(cudaEventRecord(t1, b->origin));
        BCK(cudaEventSynchronize(t1));
        float ms = 0.f;
        BCK(cudaEventElapsedTime(&ms, t0, t1));
        ms /= (float)steps;
        if (ms < best_ms) { best_ms = ms; best = k; }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    assign(b, best);
    if (chosen) *chosen = best;
    if (ms_per_step) *ms_per_step = best_ms;
    return UGKS_OK;
}

extern "C" int ugks_batch_set_streams(ugks_batch* b, int k) {
    if (!b || k < 1 || k > b->max_slots) return UGKS_EINVAL;
    assign(b, k);
    return UGKS_OK;
}

extern "C" int ugks_batch_download(ugks_batch* b, int i, double* h, double* bb, double* W) {
    if (!b || i < 0 || i >= b->n) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    const Inst& I = b->inst[i];
    const size_t S = I.S, nc = (size_t)I.P.nx * I.P.ny;
    if (h) BCK(cudaMemcpy(h, I.B[0].h, S * sizeof(double), cudaMemcpyDeviceToHost));
    if (bb) BCK(cudaMemcpy(bb, I.B[0].b, S * sizeof(double), cudaMemcpyDeviceToHost));
    if (W) BCK(cudaMemcpy(W, I.B[0].W, nc * 4 * sizeof(double), cudaMemcpyDeviceToHost));
    return UGKS_OK;
}

extern "C" int ugks_batch_upload(ugks_batch* b, int i, const double* h, const double* bb, const double* W) {
    if (!b || i < 0 || i >= b->n || !h || !bb || !W) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    Inst& I = b->inst[i];
    const size_t S = I.S, nc = (size_t)I.P.nx * I.P.ny;
    BCK(cudaMemcpy(I.B[0].h, h, S * sizeof(double), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(I.B[0].b, bb, S * sizeof(double), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(I.B[0].W, W, nc * 4 * sizeof(double), cudaMemcpyHostToDevice));
    const BSlot& Sl = b->slot[I.slot];
    BCK(cudaMemsetAsync(I.flags, 0, 4 * sizeof(unsigned), Sl.s));
    BCK(enqueue_s2cn2_prepare(I.P, I.B[0], I.T[0], I.C, Sl.s, nullptr));
    BCK(cudaStreamSynchronize(Sl.s));
    unsigned st = 0;
    BCK(cudaMemcpy(&st, I.flags + 1, sizeof st, cudaMemcpyDeviceToHost));
    return st ? UGKS_ENUMERIC : UGKS_OK;
}

extern "C" int ugks_batch_report(ugks_batch* b, int i, double* report) {
    if (!b || i < 0 || i >= b->n || !report) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    BCK(cudaMemcpy(report, b->inst[i].C.report, kCnReport * sizeof(double), cudaMemcpyDeviceToHost));
    return UGKS_OK;
}

extern "C" int ugks_batch_wall_aero(ugks_batch* b, int i, double* out) {
    if (!b || i < 0 || i >= b->n || !out) return UGKS_EINVAL;
    BCK(cudaSetDevice(b->device));
    BCK(cudaMemcpy(out, b->inst[i].B[0].wall_aero, (size_t)2 * b->inst[i].P.nx * 3 * sizeof(double),
                   cudaMemcpyDeviceToHost));
    return UGKS_OK;
}

extern "C" long long ugks_batch_launch_count(const ugks_batch* b) { return b ? b->launches : 0; }

extern "C" void* ugks_batch_stream(ugks_batch* b) { return b ? (void*)b->origin : nullptr; }
