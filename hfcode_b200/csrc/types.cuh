// Data layout and Boys function of the B200 Fock builder, shared by the
// kernels and by the host-compiled check of the generated class code.
#pragma once
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif
#include <cmath>

namespace hfgpu {

constexpr double INTTHRESH = 1e-10;     // molprops.f90:162
constexpr int NPT = 10;                 // GPU pair types SS LS LL DS DL DD PS LP PP DP
constexpr int NCLS = 55;                // quartet classes over the pair types (21 without pure p)
constexpr int BOYS_NPT = 225;           // grid T_j = j/8, j = 0..224 (T <= 28)
constexpr int BOYS_K = 8;               // Taylor terms per grid point
// one block per order M: BOYS_NPT x BOYS_K Taylor coefficients, then the
// BOYS_NPT values exp(-T_j) used by the downward recursion
constexpr int BOYS_BLK = BOYS_NPT * (BOYS_K + 1);
constexpr int BOYS_MMAX = 8;            // highest order used: (dd|dd)

// Primitive pair (one surviving primitive product of a shell pair): exponent
// sum p, centre P, K_ab = sqrt(2 pi^2.5) exp(-ab/p r^2)/p d_a d_b
// (precalc_kabs.f90:103-109) and the L-shell p/s ratios of both primitives.
struct GPrim {
    double p;
    double P[3];
    double K;
    double w1, w2;
    double pad;
};

// Shell pair in GPU orientation (larger shell first).  Primitive ib of the
// pair is entry p0 + ib * ps of the primitive-pair arrays: ps = 1 for the
// all-pairs layout, and ps = group size for the active lists, whose pairs of
// equal primitive count are interleaved so that the lanes of a warp, working
// on neighbouring pairs, read neighbouring addresses.
struct GPair {
    double A[3];
    double B[3];
    int p0, np;    // first primitive and primitive count
    int sa, sb;    // shell indices
    int aoa, aob;  // first AO of each shell
    int ps, pad;   // primitive stride
};

// Primitive pairs as four arrays of 16-byte pairs of fields of GPrim:
// (p, Px), (Py, Pz), (K, w1), (w2, 1/(2p)); one primitive pair is four
// vector loads instead of eight scalar ones.
struct alignas(16) PrimVec {
    double a, b;
};
struct PrimSoA {
    const PrimVec* v0;  // p, Px
    const PrimVec* v1;  // Py, Pz
    const PrimVec* v2;  // K, w1
    const PrimVec* v3;  // w2, 1/(2p)
};

__device__ __forceinline__ GPrim load_prim(const PrimSoA& s, int i) {
#ifdef __CUDA_ARCH__
    const double2 a = __ldg(reinterpret_cast<const double2*>(s.v0) + i);
    const double2 b = __ldg(reinterpret_cast<const double2*>(s.v1) + i);
    const double2 c = __ldg(reinterpret_cast<const double2*>(s.v2) + i);
    const double2 d = __ldg(reinterpret_cast<const double2*>(s.v3) + i);
    GPrim g;
    g.p = a.x;
    g.P[0] = a.y;
    g.P[1] = b.x;
    g.P[2] = b.y;
    g.K = c.x;
    g.w1 = c.y;
    g.w2 = d.x;
    g.pad = d.y;  // 1/(2p)
#else
    const PrimVec a = s.v0[i], b = s.v1[i], c = s.v2[i], d = s.v3[i];
    GPrim g;
    g.p = a.a;
    g.P[0] = a.b;
    g.P[1] = b.a;
    g.P[2] = b.b;
    g.K = c.a;
    g.w1 = c.b;
    g.w2 = d.a;
    g.pad = d.b;
#endif
    return g;
}

// ---------------------------------------------------------------- Boys ----
// F_m(T) for m = 0..M.  T > 28: F_0 = sqrt(pi/T)/2 and upward recursion
// without the exponential, which is what the reference evaluates there
// (boys.f90:134-139).  T <= 28: 8-term Taylor expansion of F_M about the
// nearest point of a 1/8-spaced grid (coefficients F_{M+k}(T_j)(-1)^k/k!
// staged in shared memory), then downward recursion
// F_m = (2T F_{m+1} + e^-T)/(2m+1).
template <int M>
__device__ __forceinline__ void boys_eval(double T, const double* __restrict__ tab, double* F) {
    if (T > 28.0) {
        const double rt = rsqrt(T);  // one reciprocal square root gives sqrt(1/T) and 1/T
        const double it = rt * rt;
        F[0] = 0.88622692545275801365 * rt;
#pragma unroll
        for (int m = 1; m <= M; ++m) F[m] = F[m - 1] * ((m - 0.5) * it);
    } else {
        const int j = __double2int_rn(T * 8.0);
        const double x = T - 0.125 * j;
        const double* c = tab + j * BOYS_K;
        double f = c[BOYS_K - 1];
#pragma unroll
        for (int k = BOYS_K - 2; k >= 0; --k) f = fma(f, x, c[k]);
        F[M] = f;
        if (M > 0) {
            // exp(-T) = exp(-T_j) exp(-x), |x| <= 1/16: ten Taylor terms of
            // exp(-x) leave a truncation error below 3e-19
            double ex = 1.0 / 3628800.0;
            ex = fma(ex, -x, 1.0 / 362880.0);
            ex = fma(ex, -x, 1.0 / 40320.0);
            ex = fma(ex, -x, 1.0 / 5040.0);
            ex = fma(ex, -x, 1.0 / 720.0);
            ex = fma(ex, -x, 1.0 / 120.0);
            ex = fma(ex, -x, 1.0 / 24.0);
            ex = fma(ex, -x, 1.0 / 6.0);
            ex = fma(ex, -x, 0.5);
            ex = fma(ex, -x, 1.0);
            ex = fma(ex, -x, 1.0);
            const double e = tab[BOYS_NPT * BOYS_K + j] * ex;
            const double t2 = T + T;
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * (1.0 / (2 * m + 1));
        }
    }
}

template <int M>
__device__ __forceinline__ void boys_eval(float T, const float* __restrict__ tab, float* F) {
    if (T > 28.0f) {
        const float rt = rsqrtf(T);
        const float it = rt * rt;
        F[0] = 0.886226925f * rt;
#pragma unroll
        for (int m = 1; m <= M; ++m) F[m] = F[m - 1] * ((m - 0.5f) * it);
    } else {
        const int j = __float2int_rn(T * 8.0f);
        const float x = T - 0.125f * j;
        const float* c = tab + j * BOYS_K;
        float f = c[5];
#pragma unroll
        for (int k = 4; k >= 0; --k) f = fmaf(f, x, c[k]);
        F[M] = f;
        if (M > 0) {
            const float e = __expf(-T);
            const float t2 = T + T;
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = fmaf(t2, F[m + 1], e) * (1.0f / (2 * m + 1));
        }
    }
}


}  // namespace hfgpu
