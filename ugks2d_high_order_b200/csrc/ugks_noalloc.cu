// ugks_noalloc.cu -- an Explicit-step entry point that allocates no memory at all.
//
// Who needs it: host codes that manage every byte of device memory themselves (a Fortran or
// C driver with its own pre-sized device pool, or an application running under a memory cap
// where a later cudaMalloc may fail) and latency-critical loops where cudaMalloc/cudaFree would
// implicitly synchronise the device.  Such callers cannot create a ugks_ctx, because
// ugks_ctx_create allocates the working arrays.  This entry point takes the caller's own device
// arrays for the inputs and outputs and keeps all of its working arrays (Van-Leer slopes, face
// fluxes, per-cell reductions, the status word) in one file-scope __device__ array of fixed size.
//
// Limits and behaviour (also stated in include/ugks_b200.h):
//   * The scratch array is kNoAllocBytes = 36 MiB.  A call whose working set does not fit is
//     rejected with UGKS_EINVAL before any GPU work; the reference's delivered case (8x64 cells,
//     32x32 velocities) needs 33.8 MB.  The array belongs to this file's device module.  Under
//     CUDA's lazy module loading (the default) that module, and with it the 36 MiB, is loaded on a
//     device at the first call there, so a caller that sizes its own device pool or runs under a
//     memory cap makes one call on each device before it does so.  The array then stays until the
//     process exits.
//   * The first call on a device looks the array's device address up (cudaGetSymbolAddress) with
//     that device current.
//   * Every call synchronises its stream twice: once after copying the velocity table to the host
//     (U_MAX / V_MAX set the time step) and once after reading the status and the outputs.  The
//     call therefore cannot be captured in a CUDA graph.
//   * Every call uses the same array and it keeps the previous call's contents; this call clears
//     what must start at zero (the last-CTA counter and the status word).  Calls that overlap on
//     the GPU (other streams, other host threads driving the same device) race on the array and
//     must be serialised by the caller.  Host threads that drive different devices use different
//     arrays and share no host state.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>

#include "../../include/ugks_b200.h"
#include "ugks_lo.cuh"

namespace ugks {
cudaError_t launch_lo_slopes(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_faces(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_walls(const LoParams& P, const LoBuffers& B, cudaStream_t s);
cudaError_t launch_lo_cells(const LoParams& P, const LoBuffers& B, int mode, bool collision, cudaStream_t s);
cudaError_t launch_lo_timestep(const LoParams& P, const LoBuffers& B, cudaStream_t s);
}  // namespace ugks

using namespace ugks;

namespace {

constexpr size_t kNoAllocBytes = (size_t)36 << 20;
constexpr size_t kNoAllocDoubles = kNoAllocBytes / sizeof(double);
constexpr int kMaxDevices = 64;

// The scratch.  Host code must not use this name as an address: in host code it names a
// host-side shadow, so only the address returned by cudaGetSymbolAddress is passed to kernels.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Device address of the scratch per device, filled on the first call on that device.  Every lookup of
// one device yields the same address, so two host threads filling one entry at once store the same
// value; the entries are atomic so that such a store is well defined.
std::atomic<double*> g_scratch_addr[kMaxDevices];

struct Plan {
    size_t flags, sxh, syh, sxb, syb, fxh, fxb, fxw, fyh, fyb, fyw, dtl, dt, cd, dg, wa, total;
};

Plan plan_for(int nx, int ny, int nv) {
    Plan p{};
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += (n + 31) / 32 * 32; return o; };   // 256-byte aligned
    const size_t nc = (size_t)nx * ny, S = nc * nv, SY = (size_t)(ny + 1) * nx * nv;
    p.flags = take(4);
    p.sxh = take(S); p.syh = take(S); p.sxb = take(S); p.syb = take(S);
    p.fxh = take(S); p.fxb = take(S); p.fxw = take(nc * 4);
    p.fyh = take(SY); p.fyb = take(SY); p.fyw = take((size_t)(ny + 1) * nx * 4);
    p.dtl = take(nc); p.dt = take(2); p.cd = take(nc * kNDiag); p.dg = take(kNDiag);
    p.wa = take((size_t)2 * nx * 3);
    p.total = off;
    return p;
}

int fail(cudaError_t e) {
    std::fprintf(stderr, "ugks_step_explicit_noalloc: CUDA error %s\n", cudaGetErrorString(e));
    return UGKS_ECUDA;
}

}  // namespace

extern "C" int ugks_step_explicit_noalloc(const ugks_params* prm, const double* u, const double* v, const double* w,
                                          double* h, double* b, double* W, int nsteps, void* stream,
                                          double* dt_out, double* res_out) {
    if (!prm || !u || !v || !w || !h || !b || !W || nsteps < 0) return UGKS_EINVAL;
    if (prm->method != UGKS_METHOD_EXPLICIT) return UGKS_EUNSUPPORTED;
    const int nx = prm->nx, ny = prm->ny, nv = prm->nvel;
    if (nx < 1 || ny < 3 || nv < 1 || nv > kMaxVel || !(prm->dx > 0) || !(prm->dy > 0) || prm->ck < 1)
        return UGKS_EINVAL;
    const Plan pl = plan_for(nx, ny, nv);
    if (pl.total > kNoAllocDoubles) {
        std::fprintf(stderr,
                     "ugks_step_explicit_noalloc: %dx%d cells x %d velocities need %zu bytes of scratch, "
                     "more than the fixed %zu-byte array\n",
                     nx, ny, nv, pl.total * sizeof(double), kNoAllocBytes);
        return UGKS_EINVAL;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(e);
    if (dev < 0 || dev >= kMaxDevices) return UGKS_EINVAL;
    double* base = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!base) {   // once per device, with that device current
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(e);
        base = static_cast<double*>(ptr);
        g_scratch_addr[dev].store(base, std::memory_order_release);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // U_MAX, V_MAX of the table (InitVelocityFromStructuredFile, mod_InitializeFlow.f90:508), staged in
    // this call's own stack buffers (40 KB at the largest table), so concurrent calls from other host
    // threads share no host memory
    double hu[kMaxVel], hv[kMaxVel];
    e = cudaMemcpyAsync(hu, u, nv * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hv, v, nv * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(e);
    double umax = -INFINITY, vmax = -INFINITY;
    for (int k = 0; k < nv; ++k) { umax = std::fmax(umax, hu[k]); vmax = std::fmax(vmax, hv[k]); }
    const LoParams P = make_lo_params(*prm, umax, vmax);

    LoBuffers B{};
    B.u = u; B.v = v; B.w = w; B.h = h; B.b = b; B.W = W;
    B.sxh = base + pl.sxh; B.syh = base + pl.syh; B.sxb = base + pl.sxb; B.syb = base + pl.syb;
    B.fxh = base + pl.fxh; B.fxb = base + pl.fxb; B.fxw = base + pl.fxw;
    B.fyh = base + pl.fyh; B.fyb = base + pl.fyb; B.fyw = base + pl.fyw;
    B.dtl = base + pl.dtl; B.dt = base + pl.dt; B.cell_diag = base + pl.cd; B.diag = base + pl.dg;
    B.wall_aero = base + pl.wa;
    B.counter = reinterpret_cast<unsigned*>(base + pl.flags);
    B.status = B.counter + 1;
    // the fused explicit step reads no residual cache and no collision arrays
    B.res_w = B.res_h = B.res_b = nullptr;
    B.peq_h = B.peq_b = B.pcol_h = B.pcol_b = nullptr;

    // the counter and the status word must start at zero; the previous call left its values
    e = cudaMemsetAsync(base + pl.flags, 0, 4 * sizeof(double), s);
    if (e == cudaSuccess) e = launch_lo_timestep(P, B, s);
    for (int k = 0; k < nsteps && e == cudaSuccess; ++k) {
        e = launch_lo_slopes(P, B, s);
        if (e == cudaSuccess) e = launch_lo_faces(P, B, s);
        if (e == cudaSuccess) e = launch_lo_walls(P, B, s);
        if (e == cudaSuccess) e = launch_lo_cells(P, B, 3, false, s);
    }
    if (e != cudaSuccess) return fail(e);
    unsigned status = 0;
    double dt2[2] = {0.0, 0.0}, dg[kNDiag];
    e = cudaMemcpyAsync(&status, B.status, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt2, B.dt, sizeof dt2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dg, B.diag, sizeof dg, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(e);
    if (dt_out) *dt_out = nsteps > 0 ? dt2[1] : dt2[0];
    if (res_out && nsteps > 0) finish_explicit_res(nx, ny, dg, res_out);
    return status ? UGKS_ENUMERIC : UGKS_OK;
}
