// J/K scatter of one shell quartet's ERI block held in memory with a stride
// (the staged classes' scratch), into the one-triangle buffer G
// (F += G + G^T later), one FP64 atomic per block element:
//   J_ab += 2s P_cd e,  J_cd += 2s P_ab e,
//   K_ac -= s/2 P_bd e, K_ad -= s/2 P_bc e, K_bc -= s/2 P_ad e, K_bd -= s/2 P_ac e.
// One pass over the block: the first index i is a loop, (j, k, l) are
// unrolled, so every element is read once; blocks indexed by i are flushed
// per i, the others once at the end.  Host-compilable with the shims of the
// test harness.
#pragma once
#include "types.cuh"

namespace hfgpu {

template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void scatter_strided(const double* __restrict__ e, size_t st, double s,
                                                const GPair& bra, const GPair& ket,
                                                const double* __restrict__ P, double* __restrict__ G, int nb,
                                                bool jonly) {
    const int a0 = bra.aoa, b0 = bra.aob, c0 = ket.aoa, d0 = ket.aob;
    auto Pm = [&](int r, int c) { return __ldg(P + r + (size_t)c * nb); };
    auto Ga = [&](int r, int c) { return G + r + (size_t)c * nb; };
    const double s2 = 2.0 * s, hs = -0.5 * s;
    double jcd[NC * ND], kbc[NB * NC], kbd[NB * ND], pcd[NC * ND];
#pragma unroll
    for (int x = 0; x < NC * ND; ++x) jcd[x] = 0.0;
#pragma unroll
    for (int x = 0; x < NB * NC; ++x) kbc[x] = 0.0;
#pragma unroll
    for (int x = 0; x < NB * ND; ++x) kbd[x] = 0.0;
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) pcd[k * ND + l] = Pm(c0 + k, d0 + l);
#pragma unroll 1
    for (int i = 0; i < NA; ++i) {
        double jab[NB], kac[NC], kad[ND], pad_[ND], pac[NC];
#pragma unroll
        for (int j = 0; j < NB; ++j) jab[j] = 0.0;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            kac[k] = 0.0;
            pac[k] = Pm(a0 + i, c0 + k);
        }
#pragma unroll
        for (int l = 0; l < ND; ++l) {
            kad[l] = 0.0;
            pad_[l] = Pm(a0 + i, d0 + l);
        }
        const double* ei = e + (size_t)(i * NB * NC * ND) * st;
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const double pab = Pm(a0 + i, b0 + j);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double pbc = Pm(b0 + j, c0 + k);
#pragma unroll
                for (int l = 0; l < ND; ++l) {
                    const double v = __ldg(ei + (size_t)((j * NC + k) * ND + l) * st);
                    jab[j] += pcd[k * ND + l] * v;
                    jcd[k * ND + l] += pab * v;
                    if (!jonly) {
                        kac[k] += Pm(b0 + j, d0 + l) * v;
                        kad[l] += pbc * v;
                        kbc[j * NC + k] += pad_[l] * v;
                        kbd[j * ND + l] += pac[k] * v;
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) atomicAdd(Ga(a0 + i, b0 + j), s2 * jab[j]);
        if (!jonly) {
#pragma unroll
            for (int k = 0; k < NC; ++k) atomicAdd(Ga(a0 + i, c0 + k), hs * kac[k]);
#pragma unroll
            for (int l = 0; l < ND; ++l) atomicAdd(Ga(a0 + i, d0 + l), hs * kad[l]);
        }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) atomicAdd(Ga(c0 + k, d0 + l), s2 * jcd[k * ND + l]);
    if (jonly) return;
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < NC; ++k) atomicAdd(Ga(b0 + j, c0 + k), hs * kbc[j * NC + k]);
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int l = 0; l < ND; ++l) atomicAdd(Ga(b0 + j, d0 + l), hs * kbd[j * ND + l]);
}

}  // namespace hfgpu
