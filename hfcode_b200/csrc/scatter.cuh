// J/K scatter of one shell quartet's ERI block held in memory with a stride
// (the staged classes' scratch): six two-index contractions with one P block
// each, one FP64 atomic per block element into the one-triangle buffer G
// (F += G + G^T later).  Host-compilable with the shims of the test harness.
#pragma once
#include "types.cuh"

namespace hfgpu {

template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void scatter_strided(const double* __restrict__ e, size_t st, double s,
                                                const GPair& bra, const GPair& ket,
                                                const double* __restrict__ P, double* __restrict__ G, int nb,
                                                bool jonly) {
    const int a0 = bra.aoa, b0 = bra.aob, c0 = ket.aoa, d0 = ket.aob;
    auto E = [&](int i, int j, int k, int l) {
        return __ldg(e + (size_t)(((i * NB + j) * NC + k) * ND + l) * st);
    };
    auto Pm = [&](int r, int c) { return __ldg(P + r + (size_t)c * nb); };
    auto Ga = [&](int r, int c) { return G + r + (size_t)c * nb; };
    const double s2 = 2.0 * s, hs = -0.5 * s;
    {  // J_ab <- P_cd
        double pp[NC * ND];
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
            for (int l = 0; l < ND; ++l) pp[k * ND + l] = Pm(c0 + k, d0 + l);
#pragma unroll 1
        for (int i = 0; i < NA; ++i)
#pragma unroll 1
            for (int j = 0; j < NB; ++j) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < NC; ++k)
#pragma unroll
                    for (int l = 0; l < ND; ++l) acc += pp[k * ND + l] * E(i, j, k, l);
                atomicAdd(Ga(a0 + i, b0 + j), s2 * acc);
            }
    }
    {  // J_cd <- P_ab
        double pp[NA * NB];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j) pp[i * NB + j] = Pm(a0 + i, b0 + j);
#pragma unroll 1
        for (int k = 0; k < NC; ++k)
#pragma unroll 1
            for (int l = 0; l < ND; ++l) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int j = 0; j < NB; ++j) acc += pp[i * NB + j] * E(i, j, k, l);
                atomicAdd(Ga(c0 + k, d0 + l), s2 * acc);
            }
    }
    if (jonly) return;
    {  // K_ac <- P_bd
        double pp[NB * ND];
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int l = 0; l < ND; ++l) pp[j * ND + l] = Pm(b0 + j, d0 + l);
#pragma unroll 1
        for (int i = 0; i < NA; ++i)
#pragma unroll 1
            for (int k = 0; k < NC; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < NB; ++j)
#pragma unroll
                    for (int l = 0; l < ND; ++l) acc += pp[j * ND + l] * E(i, j, k, l);
                atomicAdd(Ga(a0 + i, c0 + k), hs * acc);
            }
    }
    {  // K_ad <- P_bc
        double pp[NB * NC];
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k) pp[j * NC + k] = Pm(b0 + j, c0 + k);
#pragma unroll 1
        for (int i = 0; i < NA; ++i)
#pragma unroll 1
            for (int l = 0; l < ND; ++l) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < NB; ++j)
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc += pp[j * NC + k] * E(i, j, k, l);
                atomicAdd(Ga(a0 + i, d0 + l), hs * acc);
            }
    }
    {  // K_bc <- P_ad
        double pp[NA * ND];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int l = 0; l < ND; ++l) pp[i * ND + l] = Pm(a0 + i, d0 + l);
#pragma unroll 1
        for (int j = 0; j < NB; ++j)
#pragma unroll 1
            for (int k = 0; k < NC; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int l = 0; l < ND; ++l) acc += pp[i * ND + l] * E(i, j, k, l);
                atomicAdd(Ga(b0 + j, c0 + k), hs * acc);
            }
    }
    {  // K_bd <- P_ac
        double pp[NA * NC];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int k = 0; k < NC; ++k) pp[i * NC + k] = Pm(a0 + i, c0 + k);
#pragma unroll 1
        for (int j = 0; j < NB; ++j)
#pragma unroll 1
            for (int l = 0; l < ND; ++l) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc += pp[i * NC + k] * E(i, j, k, l);
                atomicAdd(Ga(b0 + j, d0 + l), hs * acc);
            }
    }
}

}  // namespace hfgpu
