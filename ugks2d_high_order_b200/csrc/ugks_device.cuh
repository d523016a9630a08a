// ugks_device.cuh -- FP64 device math for the UGKS kinetic hot path on sm_100a.
//
// Each helper restates one routine of the reference Fortran (file:line relative to the reference
// project root).  All arithmetic is IEEE FP64; CUDA's exp/erfc/pow are used as library calls.
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

namespace ugks {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kSMV = 1.1754943508222875e-38;   // tiny(0.0_real32): mod_Globaldata.f90:26
constexpr double kEps = DBL_EPSILON;               // epsilon(1.0_KREAL)
constexpr int kMNUM = 6;                          // mod_Evolution.f90:9
constexpr int kMTUM = 5;                          // mod_Evolution.f90:10

// Status bits written to the context's device status word (first error wins per bit).
enum : unsigned {
    ST_GETPRIMARY = 1u << 0,     // reference abort 101-103
    ST_TAU = 1u << 1,            // 104-106
    ST_FACE_PROJECTION = 1u << 2,  // 446: face-equilibrium moment projection failed
    ST_PROJECTION = 1u << 3,     // 444: cell projection failed
    ST_NONFINITE_FLUX = 1u << 4, // 13-16
    ST_NONFINITE_STATE = 1u << 5,  // 4, 17
    ST_TIMEOUT = 1u << 6,        // bounded wait expired
    ST_ALPHA = 1u << 7,          // implicit admissible alpha not found
    ST_MOMENT_GATE = 1u << 8,    // implicit moment gate (Implicit_MomentTol)
    ST_STEP_REJECTED = 1u << 9,  // 203: an S2CN2 step failed its cnres / mmerr / conservation gates
    ST_W1T_PREDICTOR = 1u << 11, // 449: the W1T midpoint predictor (or its W1D faces) failed
    ST_W2R = 1u << 12,           // 456: the W2R shared predictor or its corrected faces failed
};

struct Prim { double r, U, V, L; };   // [rho, U, V, lambda = 1/T_native]

// GetPrimary (mod_Tools.f90:209-235).  Returns false on the reference's abort conditions.
__device__ __forceinline__ bool get_primary(double gm1, const double w[4], Prim& p) {
    if (!(isfinite(w[0]) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]))) return false;
    if (w[0] <= 0.0) return false;
    double denom = w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / w[0];
    if (!isfinite(denom) || denom <= 0.0) return false;
    p.r = w[0];
    p.U = w[1] / w[0];
    p.V = w[2] / w[0];
    p.L = 0.5 * w[0] / (gm1 * denom);
    return true;
}

// GetConserved (mod_Tools.f90:190-200)
__device__ __forceinline__ void get_conserved(double gm1, const Prim& p, double w[4]) {
    w[0] = p.r;
    w[1] = p.r * p.U;
    w[2] = p.r * p.V;
    w[3] = 0.5 * p.r / (p.L * gm1) + 0.5 * p.r * (p.U * p.U + p.V * p.V);
}

// GetTau with the power-law viscosity (mod_Tools.f90:267-299)
__device__ __forceinline__ bool get_tau(double mu_ref, double omega, const Prim& p, double& tau) {
    if (!(p.r > 0.0) || !(p.L > 0.0) || !isfinite(p.r) || !isfinite(p.U) || !isfinite(p.V) || !isfinite(p.L))
        return false;
    double mu = mu_ref * pow(1.0 / p.L, omega);
    if (!isfinite(mu) || mu <= 0.0) return false;
    tau = mu / (0.5 * p.r / p.L);
    return isfinite(tau) && tau > 0.0;
}

// MicroSlope (mod_Evolution.f90:1792-1800)
__device__ __forceinline__ void micro_slope(int ck, const Prim& p, const double sw[4], double a[4]) {
    const double c2 = (double)(ck + 2);
    a[3] = 4.0 * (p.L * p.L) / (c2 * p.r) *
           (2.0 * sw[3] - 2.0 * p.U * sw[1] - 2.0 * p.V * sw[2] + sw[0] * (p.U * p.U + p.V * p.V - 0.5 * c2 / p.L));
    a[2] = 2.0 * p.L / p.r * (sw[2] - p.V * sw[0]) - p.V * a[3];
    a[1] = 2.0 * p.L / p.r * (sw[1] - p.U * sw[0]) - p.U * a[3];
    a[0] = sw[0] / p.r - p.U * a[1] - p.V * a[2] - 0.5 * (p.U * p.U + p.V * p.V + 0.5 * c2 / p.L) * a[3];
}

struct Moments {
    double Mu[kMNUM + 1], MuL[kMNUM + 1], MuR[kMNUM + 1], Mv[kMTUM + 1], Mxi[3];
};

// CalcMoment (mod_Evolution.f90:1810-1842): half-range moments use erfc.
__device__ __forceinline__ void calc_moment(int ck, const Prim& p, Moments& m) {
    const double sL = sqrt(p.L);
    const double e = 0.5 * exp(-p.L * p.U * p.U) / sqrt(kPi * p.L);
    m.MuL[0] = 0.5 * erfc(-sL * p.U);
    m.MuL[1] = p.U * m.MuL[0] + e;
    m.MuR[0] = 0.5 * erfc(sL * p.U);
    m.MuR[1] = p.U * m.MuR[0] - e;
#pragma unroll
    for (int i = 2; i <= kMNUM; ++i) {
        m.MuL[i] = p.U * m.MuL[i - 1] + 0.5 * (double)(i - 1) * m.MuL[i - 2] / p.L;
        m.MuR[i] = p.U * m.MuR[i - 1] + 0.5 * (double)(i - 1) * m.MuR[i - 2] / p.L;
    }
#pragma unroll
    for (int i = 0; i <= kMNUM; ++i) m.Mu[i] = m.MuL[i] + m.MuR[i];
    m.Mv[0] = 1.0;
    m.Mv[1] = p.V;
#pragma unroll
    for (int i = 2; i <= kMTUM; ++i) m.Mv[i] = p.V * m.Mv[i - 1] + 0.5 * (double)(i - 1) * m.Mv[i - 2] / p.L;
    m.Mxi[0] = 1.0;
    m.Mxi[1] = 0.5 * (double)ck / p.L;
    m.Mxi[2] = (double)ck * ((double)ck + 2.0) / (4.0 * p.L * p.L);
}

// Moment_uvxi (mod_Evolution.f90:1853-1862)
__device__ __forceinline__ void moment_uvxi(const double* Mu, const double* Mv, const double* Mxi, int al, int be,
                                            int de, double o[4]) {
    o[0] = Mu[al] * Mv[be] * Mxi[de / 2];
    o[1] = Mu[al + 1] * Mv[be] * Mxi[de / 2];
    o[2] = Mu[al] * Mv[be + 1] * Mxi[de / 2];
    o[3] = 0.5 * (Mu[al + 2] * Mv[be] * Mxi[de / 2] + Mu[al] * Mv[be + 2] * Mxi[de / 2] +
                  Mu[al] * Mv[be] * Mxi[(de + 2) / 2]);
}

// Moment_auvxi (mod_Evolution.f90:1874-1885)
__device__ __forceinline__ void moment_auvxi(const double a[4], const double* Mu, const double* Mv,
                                             const double* Mxi, int al, int be, double o[4]) {
    double t0[4], t1[4], t2[4], t3[4], t4[4], t5[4];
    moment_uvxi(Mu, Mv, Mxi, al, be, 0, t0);
    moment_uvxi(Mu, Mv, Mxi, al + 1, be, 0, t1);
    moment_uvxi(Mu, Mv, Mxi, al, be + 1, 0, t2);
    moment_uvxi(Mu, Mv, Mxi, al + 2, be, 0, t3);
    moment_uvxi(Mu, Mv, Mxi, al, be + 2, 0, t4);
    moment_uvxi(Mu, Mv, Mxi, al, be, 2, t5);
#pragma unroll
    for (int m = 0; m < 4; ++m)
        o[m] = a[0] * t0[m] + a[1] * t1[m] + a[2] * t2[m] + 0.5 * a[3] * t3[m] + 0.5 * a[3] * t4[m] +
               0.5 * a[3] * t5[m];
}

// Mt(1..5) (mod_Evolution.f90:346-350); Mt[0..4] here.
__device__ __forceinline__ void time_coeffs(double dt, double tau, double Mt[5]) {
    const double e = exp(-dt / tau);
    Mt[3] = tau * (1.0 - e);
    Mt[4] = -tau * dt * e + tau * Mt[3];
    Mt[0] = dt - Mt[3];
    Mt[1] = -tau * Mt[0] + Mt[4];
    Mt[2] = 0.5 * (dt * dt) - tau * Mt[0];
}

// Van-Leer limited slope (mod_Interpolation.f90:162-168)
__device__ __forceinline__ double vanleer(double sL, double sR) {
    return (copysign(1.0, sR) + copysign(1.0, sL)) * fabs(sR) * fabs(sL) / (fabs(sR) + fabs(sL) + kSMV);
}

// SolveDense4 (mod_ImplicitCommon.f90:84-113): Gauss-Jordan with partial pivoting on a
// row-major 4x4.  Returns false where the reference sets ok=.false.  The pivot row is found as in
// the reference (first row with the strictly largest |a(r,col)|) and swapped with predicated moves
// on compile-time indices, so the augmented matrix stays in registers.
__device__ __forceinline__ bool solve_dense4(const double m[16], const double rhs[4], double sol[4]) {
    double a[4][5];
    double ps = 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
        for (int c = 0; c < 4; ++c) { a[r][c] = m[r * 4 + c]; ps = fmax(ps, fabs(m[r * 4 + c])); }
        a[r][4] = rhs[r];
    }
    ps = fmax(ps, DBL_MIN);
    bool ok = true;
#pragma unroll
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        double best = fabs(a[col][col]);
#pragma unroll
        for (int r = col + 1; r < 4; ++r) {
            const double v = fabs(a[r][col]);
            if (v > best) { best = v; piv = r; }
        }
        ok = ok && !(best <= 1000.0 * kEps * ps);
#pragma unroll
        for (int r = col + 1; r < 4; ++r) {
            const bool sw = (piv == r);
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const double t = a[col][c];
                a[col][c] = sw ? a[r][c] : t;
                a[r][c] = sw ? t : a[r][c];
            }
        }
        const double d = a[col][col];
#pragma unroll
        for (int c = 0; c < 5; ++c) a[col][c] = a[col][c] / d;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (r == col) continue;
            const double f = a[r][col];
#pragma unroll
            for (int c = 0; c < 5; ++c) a[r][c] = a[r][c] - f * a[col][c];
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) { sol[r] = a[r][4]; ok = ok && isfinite(sol[r]); }
    return ok;
}

// Expand the 10 unique Gram sums (order 00,01,02,03,11,12,13,22,23,33) to a symmetric 4x4.
__device__ __forceinline__ void gram_expand(const double* g, double m[16]) {
    m[0] = g[0]; m[1] = g[1]; m[2] = g[2]; m[3] = g[3];
    m[4] = g[1]; m[5] = g[4]; m[6] = g[5]; m[7] = g[6];
    m[8] = g[2]; m[9] = g[5]; m[10] = g[7]; m[11] = g[8];
    m[12] = g[3]; m[13] = g[6]; m[14] = g[8]; m[15] = g[9];
}

// Per-velocity contribution to the ProjectToConservedMoments Gram matrix
// (mod_ImplicitCommon.f90:58-67): weight_local*(w_h*kh*kh^T + w_b*kb*kb^T), kb = (0,0,0,1/2).
__device__ __forceinline__ void gram_add(double wl, double wh, double wb, double un, double ut, double* g) {
    const double e = 0.5 * (un * un + ut * ut);
    const double a = wl * wh;
    g[0] += a;
    g[1] += a * un;
    g[2] += a * ut;
    g[3] += a * e;
    g[4] += a * un * un;
    g[5] += a * un * ut;
    g[6] += a * un * e;
    g[7] += a * ut * ut;
    g[8] += a * ut * e;
    g[9] += a * e * e + wl * wb * 0.25;
}

// MomentConserved integrand (mod_ImplicitCommon.f90:32-40)
__device__ __forceinline__ void moment_add(double wl, double un, double ut, double h, double b, double* m) {
    m[0] += wl * h;
    m[1] += wl * un * h;
    m[2] += wl * ut * h;
    m[3] += 0.5 * wl * ((un * un + ut * ut) * h + b);
}

// ---------------------------------------------------------------------------------------------
// Block-wide reductions.  NS sums followed by NM maxima (NS, NM <= 32) are reduced in a fixed
// tree, so results are deterministic run to run.  Inside a warp the values are reduced by
// recursive halving: at each xor-shuffle distance every lane keeps one half of its values and sends
// the other half, so N values cost about N shuffles instead of 5N.  Then one lane per value and
// warp writes a partial, and a serial sum over the warps finishes.  Every thread returns with the
// block totals in v[0..NS+NM).  red needs (blockDim/32)*(pow2(NS)+pow2(NM)) doubles, out NS+NM.
constexpr int pow2_ceil(int n) { return n <= 1 ? 1 : 2 * pow2_ceil((n + 1) / 2); }
constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

template <int N, bool MAX>
__device__ __forceinline__ double warp_halving(const double* v) {
    constexpr int NP = pow2_ceil(N);
    double t[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) t[i] = i < N ? v[i] : (MAX ? -INFINITY : 0.0);
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int o = 16 >> s;
        const int len = NP >> s;          // live values per lane before this step
        if (len > 1) {
            const int half = len >> 1;
            const bool up = (lane & o) != 0;
#pragma unroll
            for (int i = 0; i < half; ++i) {
                const double keep = up ? t[i + half] : t[i];
                const double send = up ? t[i] : t[i + half];
                const double recv = __shfl_xor_sync(0xffffffffu, send, o);
                t[i] = MAX ? fmax(keep, recv) : keep + recv;
            }
        } else {
            const double recv = __shfl_xor_sync(0xffffffffu, t[0], o);
            t[0] = MAX ? fmax(t[0], recv) : t[0] + recv;
        }
    }
    return t[0];   // the total of logical index (lane >> (5 - log2 NP)) when NP <= 32
}

// Warp-wide sums (maxima) of N values per lane; every lane returns with the totals in v[0..N).
template <int N>
__device__ __forceinline__ void warp_sum_all(double* v) {
    constexpr int sh = 5 - ilog2(pow2_ceil(N));
    const double r = warp_halving<N, false>(v);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __shfl_sync(0xffffffffu, r, i << sh);
}
template <int N>
__device__ __forceinline__ void warp_max_all(double* v) {
    constexpr int sh = 5 - ilog2(pow2_ceil(N));
    const double r = warp_halving<N, true>(v);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __shfl_sync(0xffffffffu, r, i << sh);
}

// Compensated summation.  two_sum (Knuth, TAOCP vol. 2, 4.2.2): s = fl(a + b) and the exact rounding error
// e = a + b - s, in either argument order.  A compensated sum carries (s, c): every term enters s through
// two_sum and its error into c (Neumaier's form of Kahan summation); the sum is s + c.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void comp_add(double& s, double& c, double x) {
    double t, e;
    two_sum(s, x, t, e);
    s = t;
    c = c + e;
}
// Warp totals of N compensated per-lane sums (s, c): an xor butterfly that joins pairs by two_sum and adds
// their compensations, so both lanes of a pair compute the same values; every lane returns the totals
// s + c in s[0..N).
template <int N>
__device__ __forceinline__ void warp_sum_all_comp(double* s, double* c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const double os = __shfl_xor_sync(0xffffffffu, s[m], o), oc = __shfl_xor_sync(0xffffffffu, c[m], o);
            double t, e;
            two_sum(s[m], os, t, e);
            s[m] = t;
            c[m] = (c[m] + oc) + e;
        }
#pragma unroll
    for (int m = 0; m < N; ++m) s[m] = s[m] + c[m];
}

// Reduce into shared memory only: on return out[0..NS+NM) holds the block totals and is visible
// to every thread.  The next reduction writes `out` only after its first barrier, which no thread
// passes before it has read this one, so no trailing barrier is needed.
template <int NS, int NM>
__device__ __forceinline__ void block_reduce_smem(const double* v, double* red, double* out) {
    constexpr int PS = NS > 0 ? pow2_ceil(NS) : 0;
    constexpr int PM = NM > 0 ? pow2_ceil(NM) : 0;
    constexpr int W = PS + PM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (NS > 0) {
        const double r = warp_halving<NS, false>(v);
        constexpr int sh = 5 - ilog2(PS);
        if ((lane & ((1 << sh) - 1)) == 0) red[warp * W + (lane >> sh)] = r;
    }
    if (NM > 0) {
        const double r = warp_halving<NM, true>(v + NS);
        constexpr int sh = 5 - ilog2(PM);
        if ((lane & ((1 << sh) - 1)) == 0) red[warp * W + PS + (lane >> sh)] = r;
    }
    __syncthreads();
    if (threadIdx.x < NS + NM) {
        const int i = threadIdx.x;
        const int col = i < NS ? i : PS + (i - NS);
        double s = red[col];
        if (i < NS) { for (int w = 1; w < nw; ++w) s += red[w * W + col]; }
        else { for (int w = 1; w < nw; ++w) s = fmax(s, red[w * W + col]); }
        out[i] = s;
    }
    __syncthreads();
}

template <int NS, int NM>
__device__ __forceinline__ void block_reduce(double* v, double* red, double* out) {
    block_reduce_smem<NS, NM>(v, red, out);
#pragma unroll
    for (int i = 0; i < NS + NM; ++i) v[i] = out[i];
}

__device__ __forceinline__ void set_status(unsigned* status, unsigned bit) {
    atomicOr(status, bit);
}

}  // namespace ugks
