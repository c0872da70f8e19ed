// Shared device code of the B200 Fock builder: data layout, Boys function,
// J/K scatter and the kernel templates instantiated once per quartet class
// (one translation unit per class, see generated/cls_*.cu).
#pragma once
#include <cuda_runtime.h>

#include "types.cuh"
#include "scatter.cuh"

#include <cstdint>
#include <type_traits>

namespace hfgpu {

// ------------------------------------------------------- class traits ----
// functions of the first / second shell of pair type t
// (SS LS LL DS DL DD PS LP PP DP)
__host__ __device__ constexpr int pt_na(int t) {
    return t == 0 ? 1 : t <= 2 ? 4 : t <= 5 ? 5 : t == 6 ? 3 : t == 7 ? 4 : t == 8 ? 3 : 5;
}
__host__ __device__ constexpr int pt_nb(int t) {
    return t == 0 || t == 1 || t == 3 || t == 6 ? 1 : t == 2 || t == 4 ? 4 : t == 5 ? 5 : 3;
}

#define HF_CLASS_TRAITS(ci, bi, ki, NAME, nout, L)                                                   \
    struct Cls_##NAME {                                                                              \
        static constexpr int CI = ci, BI = bi, KI = ki, NOUT = nout, LL = L;                         \
        __device__ __forceinline__ static void eri(const GPair& b, const GPair& k, const PrimSoA& p, \
                                                   const double* t, double* o) {                     \
            eri_##NAME(b, k, p, t, o);                                                               \
        }                                                                                            \
        __device__ __forceinline__ static void eri32(const GPair& b, const GPair& k, const PrimSoA& p, \
                                                     const float* t, float* o) {                     \
            eri_##NAME##_f32(b, k, p, t, o);                                                         \
        }                                                                                            \
    };

// ------------------------------------------------------------ scatter ----
// F contributions of one shell quartet with uniform weight s, into the
// one-triangle buffer G (F += G + G^T later).  Column-major P(r,c)=P[r+c*nb].
template <int NA, int NB, int NC, int ND, typename E>
__device__ __forceinline__ void scatter_quartet(const E* e, double s, int a0, int b0, int c0, int d0,
                                                const double* __restrict__ P, double* __restrict__ G,
                                                int nb, bool jonly) {
    auto Pm = [&](int r, int c) { return __ldg(P + r + (size_t)c * nb); };
    auto idx = [](int i, int j, int k, int l) { return ((i * NB + j) * NC + k) * ND + l; };
    double pcd[NC * ND], pab[NA * NB];
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) pcd[k * ND + l] = Pm(c0 + k, d0 + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) pab[i * NB + j] = Pm(a0 + i, b0 + j);
    const double s2 = 2.0 * s;
    // J_ab and J_cd
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < NC; ++k)
#pragma unroll
                for (int l = 0; l < ND; ++l) acc += pcd[k * ND + l] * (double)e[idx(i, j, k, l)];
            atomicAdd(G + (a0 + i) + (size_t)(b0 + j) * nb, s2 * acc);
        }
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < NA; ++i)
#pragma unroll
                for (int j = 0; j < NB; ++j) acc += pab[i * NB + j] * (double)e[idx(i, j, k, l)];
            atomicAdd(G + (c0 + k) + (size_t)(d0 + l) * nb, s2 * acc);
        }
    if (jonly) return;
    const double hs = -0.5 * s;
    // K_ac (sum over j,l of P_jl), K_ad (P_jk), K_bc (P_il), K_bd (P_ik)
    {
        double pbd[NB * ND];
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int l = 0; l < ND; ++l) pbd[j * ND + l] = Pm(b0 + j, d0 + l);
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < NB; ++j)
#pragma unroll
                    for (int l = 0; l < ND; ++l) acc += pbd[j * ND + l] * (double)e[idx(i, j, k, l)];
                atomicAdd(G + (a0 + i) + (size_t)(c0 + k) * nb, hs * acc);
            }
    }
    {
        double pbc[NB * NC];
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k) pbc[j * NC + k] = Pm(b0 + j, c0 + k);
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int l = 0; l < ND; ++l) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < NB; ++j)
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc += pbc[j * NC + k] * (double)e[idx(i, j, k, l)];
                atomicAdd(G + (a0 + i) + (size_t)(d0 + l) * nb, hs * acc);
            }
    }
    {
        double pad_[NA * ND];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int l = 0; l < ND; ++l) pad_[i * ND + l] = Pm(a0 + i, d0 + l);
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int l = 0; l < ND; ++l) acc += pad_[i * ND + l] * (double)e[idx(i, j, k, l)];
                atomicAdd(G + (b0 + j) + (size_t)(c0 + k) * nb, hs * acc);
            }
    }
    {
        double pac[NA * NC];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int k = 0; k < NC; ++k) pac[i * NC + k] = Pm(a0 + i, c0 + k);
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int l = 0; l < ND; ++l) {
                double acc = 0.0;
#pragma unroll
                for (int i = 0; i < NA; ++i)
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc += pac[i * NC + k] * (double)e[idx(i, j, k, l)];
                atomicAdd(G + (b0 + j) + (size_t)(d0 + l) * nb, hs * acc);
            }
    }
}

// ------------------------------------------------------- kernel args ----
struct ClassStats {
    unsigned long long scattered, prim, fp32;
};

struct NDArgs {
    const uint2* quartets;  // this class's list: FP64 entries, then FP32 entries
    int n;                  // number of quartets to process (ncls == nullptr)
    // Device-side counts [2 * NCLS] (FP64, FP32 per class) written by the
    // screen; when set, the count is ncls[2*cls+prec] and the FP32 entries
    // start after the class's ncls[2*cls] FP64 entries, so the launch needs
    // no host round trip and can be captured in a CUDA graph.
    const unsigned long long* ncls;
    int cls, prec;
    const GPair* bra;
    const GPair* ket;
    PrimSoA prims;
    const double* boys;     // global table, [M][225][8]
    const float* boysf;
    const double* P;
    double* G;
    int nb;
    double thr;
    int jonly;
    ClassStats* stats;
};

template <int M, typename T>
__device__ __forceinline__ void stage_boys(T* sm, const T* g) {
    const T* src = g + (size_t)M * BOYS_BLK;
    for (int i = threadIdx.x; i < BOYS_BLK; i += blockDim.x) sm[i] = src[i];
    __syncthreads();
}

__device__ __forceinline__ void warp_add_stats(ClassStats* st, unsigned long long sc, unsigned long long pr,
                                               unsigned long long f32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sc += __shfl_down_sync(0xffffffffu, sc, o);
        pr += __shfl_down_sync(0xffffffffu, pr, o);
        f32 += __shfl_down_sync(0xffffffffu, f32, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (sc) atomicAdd(&st->scattered, sc);
        if (pr) atomicAdd(&st->prim, pr);
        if (f32) atomicAdd(&st->fp32, f32);
    }
}

constexpr int ND_THREADS = 128;
// Threads per block of the staged role kernels, a divisor of ND_THREADS.
// Smaller blocks at the same registers per thread (more blocks per SM) let
// the role kernels of one class stream and the scatters of another share
// the SMs at a finer grain.  C60 FP64 build: 197.6 ms with 128 threads,
// 194.1 with 64, 192.7 with 32; all-FP32 build 124.8, 122.3, 122.3 ms.
#ifndef HF_RB_THREADS
#define HF_RB_THREADS 32
#endif
constexpr int RB_THREADS = HF_RB_THREADS, RB_SCALE = ND_THREADS / RB_THREADS;
static_assert(RB_THREADS * RB_SCALE == ND_THREADS, "role blocks tile a scratch tile exactly");

template <class C, bool F32>
__global__ void __launch_bounds__(ND_THREADS) k_nondiag(NDArgs a) {
    using Real = typename std::conditional<F32, float, double>::type;
    __shared__ Real sboys[BOYS_BLK];
    if constexpr (F32) stage_boys<C::LL>(sboys, a.boysf);
    else stage_boys<C::LL>(sboys, a.boys);
    constexpr int NA = pt_na(C::BI), NB = pt_nb(C::BI), NC = pt_na(C::KI), ND = pt_nb(C::KI);
    static_assert(NA * NB * NC * ND == C::NOUT, "class size");
    unsigned long long nsc = 0, npr = 0;
    const int stride = gridDim.x * blockDim.x;
    int n = a.n;
    const uint2* quartets = a.quartets;
    if (a.ncls) {
        n = (int)a.ncls[2 * a.cls + a.prec];
        if (a.prec) quartets += a.ncls[2 * a.cls];
    }
    // every thread runs the same number of loop trips so the warp-level
    // statistics reduction below sees all 32 lanes
    const int trips = (n + stride - 1) / stride;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < trips; ++it, t += stride) {
        if (t >= n) continue;
        const uint2 q = quartets[t];
        const GPair bra = a.bra[q.x];
        const GPair ket = a.ket[q.y];
        Real e[C::NOUT];
        if constexpr (F32) C::eri32(bra, ket, a.prims, sboys, e);
        else C::eri(bra, ket, a.prims, sboys, e);
        npr += (unsigned long long)(bra.np * ket.np);
        Real mx = 0;
#pragma unroll
        for (int i = 0; i < C::NOUT; ++i) mx = fmax(mx, fabs(e[i]));
        if ((double)mx < a.thr) continue;  // fock_build_non_diag.f90:69
        ++nsc;
        const double s = (bra.sa == bra.sb ? 0.5 : 1.0) * (ket.sa == ket.sb ? 0.5 : 1.0);
        scatter_quartet<NA, NB, NC, ND>(e, s, bra.aoa, bra.aob, ket.aoa, ket.aob, a.P, a.G, a.nb, a.jonly);
    }
    if (a.stats) warp_add_stats(a.stats, nsc, npr, F32 ? nsc : 0ull);
}

struct DiagArgs {
    const GPair* pairs;
    int n;
    PrimSoA prims;
    const double* boys;
    double* schw;          // mode 0: written; mode 1: read
    const double* md;      // mode 1: nsh x nsh maxdm
    int nsh;
    const double* P;
    double* G;
    int nb;
    double thr;
};

// Shell pairs with themselves, (ab|ab): fock_build_initial_diag.f90 (MODE 0)
// and fock_build_diag.f90 (MODE 1).
template <class C, int MODE>
__global__ void __launch_bounds__(ND_THREADS) k_diag(DiagArgs a) {
    __shared__ double sboys[BOYS_BLK];
    stage_boys<C::LL>(sboys, a.boys);
    constexpr int NA = pt_na(C::BI), NB = pt_nb(C::BI);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const GPair pr = a.pairs[t];
    if (MODE == 1) {
        const double mv = fmax(a.md[pr.sa * a.nsh + pr.sb],
                               fmax(0.25 * a.md[pr.sb * a.nsh + pr.sb], 0.25 * a.md[pr.sa * a.nsh + pr.sa]));
        const double sw = a.schw[t];
        if (sw * sw * mv < a.thr) return;  // fock_build_diag.f90:20-21
    }
    double e[C::NOUT];
    C::eri(pr, pr, a.prims, sboys, e);
    if (MODE == 0) {
        double mx = 0;
#pragma unroll
        for (int i = 0; i < C::NOUT; ++i) mx = fmax(mx, fabs(e[i]));
        a.schw[t] = sqrt(mx);
    }
#pragma unroll
    for (int i = 0; i < C::NOUT; ++i)
        if (!(fabs(e[i]) > INTTHRESH)) e[i] = 0.0;  // element skip
    const double f = pr.sa == pr.sb ? 1.0 : 2.0;
    scatter_quartet<NA, NB, NA, NB>(e, f * f / 8.0, pr.aoa, pr.aob, pr.aoa, pr.aob, a.P, a.G, a.nb, false);
}


// Arguments of the staged classes' kernels: a chunk of the class's quartet
// list, and the scratch it goes through (accumulators, outputs and the
// per-role maxima, each in tiles of TQ quartets: see tcol below).
struct StagedArgs {
    const uint2* quartets;
    int n;                 // quartets in this chunk (an upper bound when ncls is set)
    long long q0;          // chunk start within the list
    const unsigned long long* ncls;  // device-side counts, as in NDArgs (or nullptr)
    int cls, prec;
    const GPair* bra;
    const GPair* ket;
    PrimSoA prims;
    const double* boys;
    const float* boysf;
    double* acc;
    double* out;
    double* mx;
    size_t stride;         // chunk capacity in quartets (a multiple of the tile size TQ)
    int nroles;            // rows of mx
    const double* P;
    double* G;
    int nb;
    double thr;
    int jonly;
    int f32;
    ClassStats* stats;
    const double* Pb;      // density in shell-pair blocks (staged scatter)
    const int* boff;       // block offsets, nsh x nsh
    // diagonal builders only
    double* schw;          // per pair (MODE 0 writes, MODE 1 reads)
    const double* md;      // nsh x nsh density maxima
    int nsh;
};

// Quartets of this chunk: a.n, or with device-side counts the part of the
// list left after q0, at most a.n.
__device__ __forceinline__ int staged_count(const StagedArgs& a) {
    if (!a.ncls) return a.n;
    const long long left = (long long)a.ncls[2 * a.cls + a.prec] - a.q0;
    return (int)(left < 0 ? 0 : left < a.n ? left : a.n);
}

// Scratch layout of a chunk.  Each region (accumulators, outputs, role
// maxima) is a sequence of tiles of TQ quartets; a tile holds the region's R
// rows of its quartets, row-major: element (row, t) sits at
// tcol(t, R) + row * TQ.  A block of ND_THREADS = TQ threads then reads and
// writes one contiguous span of R * TQ elements (a few hundred KB, within
// one or two pages), instead of R rows as far apart as the chunk is long.
constexpr int TQ = 128;
static_assert(TQ == ND_THREADS, "a block of the staged kernels covers one scratch tile");
__device__ __forceinline__ size_t tcol(int t, int R) { return (size_t)(t / TQ) * R * TQ + (t % TQ); }

__device__ __forceinline__ uint2 staged_quartet(const StagedArgs& a, int t) {
    const long long i = a.q0 + t + (a.ncls && a.prec ? (long long)a.ncls[2 * a.cls] : 0);
    return a.quartets[i];
}

// ------------------------------------------- staged scatter, async loads ----
// The staged scatter reads each quartet's ERI block (its column of the
// chunk's output tile) once.  With ~255 registers per thread only 8 warps fit on an
// SM, too few to hide the latency of plain loads, so the block's rows are
// streamed into shared memory with per-thread cp.async copies: slab s (the
// NC*ND rows of one (i, j)) is consumed while slabs s+1 .. s+NBUF-1 are in
// flight.  Every thread copies and reads only its own column, so no block
// barrier is needed; cp.async.wait_group bounds each wait by the thread's own
// copies.  P_bc and P_bd, needed for every i, are staged once in shared
// memory as well.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename E>
__device__ __forceinline__ void cp_async_elem(E* dst, const E* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(E) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
}

// Shared-memory plan of the async scatter (element size es): three slab
// buffers when they fit two blocks per SM, else two.
__host__ __device__ constexpr int scat_nbuf(int NA, int NB, int NC, int ND, int es = 8) {
    return (3 * NC * ND + NB * (NC + ND)) * ND_THREADS * es <= 110 * 1024 ? 3 : 2;
}
__host__ __device__ constexpr int scat_smem_bytes(int NA, int NB, int NC, int ND, int es = 8) {
    return (scat_nbuf(NA, NB, NC, ND, es) * NC * ND + NB * (NC + ND)) * ND_THREADS * es;
}

// E is the element type of the scratch rows and of the block sums: double
// for FP64 quartets, float for the FP32 quartets of the mixed form (their
// integrals are FP32 already; the sums go into G with FP64 atomics).
template <int NA, int NB, int NC, int ND, typename E>
__device__ __forceinline__ void scatter_async(const E* __restrict__ e, size_t st, double s, const GPair& bra,
                                              const GPair& ket, const double* __restrict__ Pb,
                                              const int* __restrict__ boff, int nsh,
                                              double* __restrict__ G, int nb, bool jonly, bool act, E* sm) {
    constexpr int T = ND_THREADS, SLAB = NC * ND, NS = NA * NB;
    constexpr int NBUF = scat_nbuf(NA, NB, NC, ND, (int)sizeof(E));
    const int tid = threadIdx.x;
    const int a0 = bra.aoa, b0 = bra.aob, c0 = ket.aoa, d0 = ket.aob;
    // density blocks in shell-pair order (row-major within a block), so each
    // row a thread reads is contiguous instead of one access per column
    const double* __restrict__ Bab = Pb + __ldg(boff + bra.sa * nsh + bra.sb);
    const double* __restrict__ Bac = Pb + __ldg(boff + bra.sa * nsh + ket.sa);
    const double* __restrict__ Bad = Pb + __ldg(boff + bra.sa * nsh + ket.sb);
    const double* __restrict__ Bbc = Pb + __ldg(boff + bra.sb * nsh + ket.sa);
    const double* __restrict__ Bbd = Pb + __ldg(boff + bra.sb * nsh + ket.sb);
    const double* __restrict__ Bcd = Pb + __ldg(boff + ket.sa * nsh + ket.sb);
    auto Ga = [&](int r, int c) { return G + r + (size_t)c * nb; };
    // The quartets of a warp are consecutive entries of a compacted list:
    // they mostly share their bra pair, and the active lists are ordered by
    // first shell within each primitive-count group, so they mostly share the
    // ket's first shell too.  A block element whose row and column shells are
    // the same in every lane has one address for the whole warp: its sums are
    // reduced across the warp and added with one atomic.
    const int lane = threadIdx.x & 31;
    auto same = [](int x) { return __all_sync(0xffffffffu, x == __shfl_sync(0xffffffffu, x, 0)); };
    const bool ua = same(a0), ub = same(b0), uc = same(c0), ud = same(d0);
    const bool wuni = ua && ub;
    // every lane calls this with the same `uni` (lanes without a quartet add 0)
    auto emit = [&](double* addr, double v, bool uni) {
        if (uni) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(addr, v);
        } else if (act) {
            atomicAdd(addr, v);
        }
    };
    E* eb = sm + tid;                      // [NBUF][SLAB][T], this thread's column
    E* pk = sm + NBUF * SLAB * T + tid;    // [NB*NC] P_bc then [NB*ND] P_bd
    auto issue = [&](int slab) {
        if (slab < NS) {
            const E* src = e + (size_t)slab * SLAB * st;
            E* dst = eb + (slab % NBUF) * SLAB * T;
#pragma unroll
            for (int r = 0; r < SLAB; ++r) cp_async_elem(dst + r * T, src + (size_t)r * st);
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
#pragma unroll
    for (int q = 0; q < NBUF - 1; ++q) issue(q);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
#pragma unroll
        for (int k = 0; k < NC; ++k) pk[(j * NC + k) * T] = (E)__ldg(Bbc + j * NC + k);
#pragma unroll
        for (int l = 0; l < ND; ++l) pk[(NB * NC + j * ND + l) * T] = (E)__ldg(Bbd + j * ND + l);
    }
    const E s2 = (E)(2.0 * s), hs = (E)(-0.5 * s);
    E jcd[NC * ND], kbc[NB * NC], kbd[NB * ND], pcd[NC * ND];
#pragma unroll
    for (int x = 0; x < NC * ND; ++x) jcd[x] = 0;
#pragma unroll
    for (int x = 0; x < NB * NC; ++x) kbc[x] = 0;
#pragma unroll
    for (int x = 0; x < NB * ND; ++x) kbd[x] = 0;
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) pcd[k * ND + l] = (E)__ldg(Bcd + k * ND + l);
#pragma unroll 1
    for (int i = 0; i < NA; ++i) {
        E jab[NB], kac[NC], kad[ND], pad_[ND], pac[NC];
#pragma unroll
        for (int j = 0; j < NB; ++j) jab[j] = 0;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            kac[k] = 0;
            pac[k] = (E)__ldg(Bac + i * NC + k);
        }
#pragma unroll
        for (int l = 0; l < ND; ++l) {
            kad[l] = 0;
            pad_[l] = (E)__ldg(Bad + i * ND + l);
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const int slab = i * NB + j;
            issue(slab + NBUF - 1);
            cp_async_wait<NBUF - 1>();  // this thread's copies of `slab` have landed
            const E* es = eb + (slab % NBUF) * SLAB * T;
            const E pab = (E)__ldg(Bab + i * NB + j);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const E pbc = pk[(j * NC + k) * T];
#pragma unroll
                for (int l = 0; l < ND; ++l) {
                    const E v = es[(k * ND + l) * T];
                    jab[j] += pcd[k * ND + l] * v;
                    jcd[k * ND + l] += pab * v;
                    if (!jonly) {
                        kac[k] += pk[(NB * NC + j * ND + l) * T] * v;
                        kad[l] += pbc * v;
                        kbc[j * NC + k] += pad_[l] * v;
                        kbd[j * ND + l] += pac[k] * v;
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) emit(Ga(a0 + i, b0 + j), act ? (double)(s2 * jab[j]) : 0.0, wuni);
        if (!jonly) {
#pragma unroll
            for (int k = 0; k < NC; ++k) emit(Ga(a0 + i, c0 + k), act ? (double)(hs * kac[k]) : 0.0, ua && uc);
#pragma unroll
            for (int l = 0; l < ND; ++l) emit(Ga(a0 + i, d0 + l), act ? (double)(hs * kad[l]) : 0.0, ua && ud);
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l)
            emit(Ga(c0 + k, d0 + l), act ? (double)(s2 * jcd[k * ND + l]) : 0.0, uc && ud);
    if (jonly) return;
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < NC; ++k)
            emit(Ga(b0 + j, c0 + k), act ? (double)(hs * kbc[j * NC + k]) : 0.0, ub && uc);
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int l = 0; l < ND; ++l)
            emit(Ga(b0 + j, d0 + l), act ? (double)(hs * kbd[j * ND + l]) : 0.0, ub && ud);
}

// Post-screen (max |e| over all roles < thr, fock_build_non_diag.f90:69) and
// J/K scatter of a staged chunk, one thread per quartet.  E is the element
// type of the chunk's output rows (float for the FP32 chunks of staged2
// classes in the mixed form).
template <int NA, int NB, int NC, int ND, typename E = double>
__global__ void __launch_bounds__(ND_THREADS, sizeof(E) == 4 ? 3 : 2) k_scatter_staged(StagedArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int cnt = staged_count(a);
    const int w0 = t - (threadIdx.x & 31);  // first quartet of this warp
    if (w0 >= cnt) return;                  // a warp with no quartet (whole warps only)
    // every lane of the warp runs the scatter so that the J_ab sums can be
    // reduced across the warp; a lane past the end works on the warp's first
    // quartet and writes nothing
    const bool valid = t < cnt;
    const int tq = valid ? t : w0;
    double m = 0.0;
    const double* __restrict__ mxc = a.mx + tcol(tq, a.nroles);
    for (int r = 0; r < a.nroles; ++r) m = fmax(m, mxc[r * TQ]);
    const uint2 q = staged_quartet(a, tq);
    const GPair bra = a.bra[q.x];
    const GPair ket = a.ket[q.y];
    const bool act = valid && !(m < a.thr);  // fock_build_non_diag.f90:69
    const unsigned long long nsc = act ? 1ull : 0ull;
    const unsigned long long npr = valid ? (unsigned long long)(bra.np * ket.np) : 0ull;
    const double s = (bra.sa == bra.sb ? 0.5 : 1.0) * (ket.sa == ket.sb ? 0.5 : 1.0);
    extern __shared__ __align__(16) double hf_scat_smem[];
    scatter_async<NA, NB, NC, ND, E>(reinterpret_cast<const E*>(a.out) + tcol(tq, NA * NB * NC * ND), TQ, s, bra,
                                     ket, a.Pb, a.boff,
                                     a.nsh, a.G, a.nb, a.jonly != 0, act, reinterpret_cast<E*>(hf_scat_smem));
    if (a.stats) warp_add_stats(a.stats, nsc, npr, a.f32 ? nsc : 0ull);
}

// ------------------------------------- grouped staged scatter (4 lanes) ----
// One quartet per group of SG = 4 lanes.  Lane g owns function g of one bra
// shell O (S = 0: the first bra shell a, S = 1: the second, b), which has
// four functions; X is the other bra shell.  The lane reads the rows of its
// NX slabs (o = g, x = 0..NX-1), each NC*ND rows, and forms
//   complete over the quartet:  J_OX[g][x] (P_cd), K_Oc[g][k] (P_Xd), K_Od[g][l] (P_Xc)
//   summed over the group:      K_Xc[x][k] (P_Od), K_Xd[x][l] (P_Oc) after slab x,
//                               J_cd[k][l] (P_OX) after the last slab
// Group sums are two-step reduce-scatters (xor 1, xor 2), so each lane adds a
// quarter of them and a quartet still issues one atomic per block element.
// Against the one-thread scatter a thread holds about a third of the block
// sums, which leaves room for more warps per SM to hide the latency of the
// row and density loads.
constexpr int SG = 4;
__host__ __device__ constexpr int scatg_smem_bytes(int NX, int NC, int ND, int es) {
    // two slab buffers of NC*ND rows per thread, then P_cd, P_Xc and P_Xd of
    // each quartet of the block ([value][quartet])
    return 2 * NC * ND * ND_THREADS * es + (NC * ND + NX * (NC + ND)) * (ND_THREADS / SG) * es;
}
// blocks per SM: as many as the shared memory allows, at most SCATG_BLK64
// for FP64 sums and four for FP32 sums (128 registers)
#ifndef SCATG_BLK64
#define SCATG_BLK64 3
#endif
__host__ __device__ constexpr int scatg_cap(int es) { return es == 8 ? SCATG_BLK64 : 4; }
__host__ __device__ constexpr int scatg_minb(int NX, int NC, int ND, int es) {
    return 225 * 1024 / scatg_smem_bytes(NX, NC, ND, es) < scatg_cap(es) ? 225 * 1024 / scatg_smem_bytes(NX, NC, ND, es)
                                                                         : scatg_cap(es);
}

// Sum N values over the four lanes of a group (reduce-scatter): on return
// v[0 .. N/4) hold the group sums of elements base .. base + N/4 of the
// input, base = (g&1 ? N/2 : 0) + (g&2 ? N/4 : 0).  N is a multiple of 4.
template <int N, typename E>
__device__ __forceinline__ int group_reduce_scatter(E* v, int g) {
    constexpr int H1 = N / 2, H2 = N / 4;
    const bool b0 = g & 1, b1 = g & 2;
#pragma unroll
    for (int i = 0; i < H1; ++i) {
        const E lo = v[i], hi = v[H1 + i];
        v[i] = (b0 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b0 ? lo : hi, 1);
    }
#pragma unroll
    for (int i = 0; i < H2; ++i) {
        const E lo = v[i], hi = v[H2 + i];
        v[i] = (b1 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b1 ? lo : hi, 2);
    }
    return (b0 ? H1 : 0) + (b1 ? H2 : 0);
}

template <int NA, int NB, int NC, int ND, int S, typename E = double>
__global__ void __launch_bounds__(ND_THREADS, scatg_minb(S == 0 ? NB : NA, NC, ND, (int)sizeof(E)))
    k_scatter_grouped(StagedArgs a) {
    constexpr int T = ND_THREADS, QB = T / SG, SLAB = NC * ND, NBUF = 2;
    constexpr int NO = S == 0 ? NA : NB, NX = S == 0 ? NB : NA;
    static_assert(NO == SG, "the lane-owned shell has four functions");
    constexpr int NK = NC + ND, NK4 = (NK + 3) / 4 * 4;  // K_Xc[x], K_Xd[x] of one slab
    constexpr int NJ4 = (NC * ND + 3) / 4 * 4;           // J_cd
    constexpr int NPS = NC * ND + NX * NK;               // density values in shared memory
    const int tid = threadIdx.x, lane = tid & 31, g = tid & (SG - 1), ql = tid / SG;
    const int cnt = staged_count(a);
    const int qi = blockIdx.x * QB + ql;
    const int w0 = blockIdx.x * QB + (tid - lane) / SG;  // first quartet of this warp
    if (w0 >= cnt) return;                              // whole warps only
    // a group past the end works on the warp's first quartet and writes nothing
    const bool valid = qi < cnt;
    const int tq = valid ? qi : w0;
    double mxq = 0.0;
    const double* __restrict__ mxc = a.mx + tcol(tq, a.nroles);
    for (int r = 0; r < a.nroles; ++r) mxq = fmax(mxq, mxc[r * TQ]);
    const uint2 q = staged_quartet(a, tq);
    const GPair bra = a.bra[q.x];
    const GPair ket = a.ket[q.y];
    const bool act = valid && !(mxq < a.thr);  // fock_build_non_diag.f90:69
    const bool jonly = a.jonly != 0;
    const int nsh = a.nsh;
    const int sO = S == 0 ? bra.sa : bra.sb, sX = S == 0 ? bra.sb : bra.sa;
    const int O0 = S == 0 ? bra.aoa : bra.aob, X0 = S == 0 ? bra.aob : bra.aoa;
    const int c0 = ket.aoa, d0 = ket.aob;
    // density blocks in shell-pair order, row-major within a block
    const double* __restrict__ Pb = a.Pb;
    const double* __restrict__ Bab = Pb + __ldg(a.boff + bra.sa * nsh + bra.sb);
    const double* __restrict__ BOc = Pb + __ldg(a.boff + sO * nsh + ket.sa);
    const double* __restrict__ BOd = Pb + __ldg(a.boff + sO * nsh + ket.sb);
    const double* __restrict__ BXc = Pb + __ldg(a.boff + sX * nsh + ket.sa);
    const double* __restrict__ BXd = Pb + __ldg(a.boff + sX * nsh + ket.sb);
    const double* __restrict__ Bcd = Pb + __ldg(a.boff + ket.sa * nsh + ket.sb);
    extern __shared__ __align__(16) double hf_scatg_smem[];
    E* eb = reinterpret_cast<E*>(hf_scatg_smem) + tid;                 // [NBUF][SLAB][T], own column
    E* sp = reinterpret_cast<E*>(hf_scatg_smem) + NBUF * SLAB * T + ql;  // [NPS][QB]: P_cd, P_Xc, P_Xd
    const E* __restrict__ e = reinterpret_cast<const E*>(a.out) + tcol(tq, NA * NB * NC * ND);
    const size_t st = TQ;
    auto issue = [&](int x) {
        if (x < NX) {
            const E* src = e + (size_t)((S == 0 ? g * NB + x : x * NB + g) * SLAB) * st;
            E* dst = eb + (x % NBUF) * SLAB * T;
#pragma unroll
            for (int r = 0; r < SLAB; ++r) cp_async_elem(dst + r * T, src + (size_t)r * st);
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
    issue(0);
    // the quartet's P_cd, P_Xc and P_Xd, loaded once by its four lanes
    for (int v = g; v < NPS; v += SG)
        sp[v * QB] = (E)__ldg(v < SLAB ? Bcd + v : v < SLAB + NX * NC ? BXc + (v - SLAB) : BXd + (v - SLAB - NX * NC));
    E poc[NC], pod[ND], pox[NX];
#pragma unroll
    for (int k = 0; k < NC; ++k) poc[k] = (E)__ldg(BOc + g * NC + k);
#pragma unroll
    for (int l = 0; l < ND; ++l) pod[l] = (E)__ldg(BOd + g * ND + l);
#pragma unroll
    for (int x = 0; x < NX; ++x) pox[x] = (E)__ldg(Bab + (S == 0 ? g * NB + x : x * NB + g));
    __syncwarp();
    // warp-uniform shells: a block element with one address for the whole
    // warp is summed over the warp's eight quartets and added by one lane
    auto same = [](int x) { return __all_sync(0xffffffffu, x == __shfl_sync(0xffffffffu, x, 0)); };
    const bool ua = same(bra.aoa), ub = same(bra.aob), uc = same(c0), ud = same(d0);
    const bool uO = S == 0 ? ua : ub, uX = S == 0 ? ub : ua;
    auto Ga = [&](int r, int c) { return a.G + r + (size_t)c * a.nb; };
    // `shuf` is warp-uniform (every lane runs the shuffles); `uni` may differ
    // between lanes of different g but is the same for lanes of equal g,
    // which are the lanes the shuffles sum over
    auto emit = [&](double* addr, double v, bool shuf, bool uni, bool has) {
        double r = v;
        if (shuf) {
            r += __shfl_xor_sync(0xffffffffu, r, 4);
            r += __shfl_xor_sync(0xffffffffu, r, 8);
            r += __shfl_xor_sync(0xffffffffu, r, 16);
        }
        if (uni) {
            if (lane < SG && has) atomicAdd(addr, r);
        } else if (act && has) {
            atomicAdd(addr, v);
        }
    };
    const double s = (bra.sa == bra.sb ? 0.5 : 1.0) * (ket.sa == ket.sb ? 0.5 : 1.0);
    const double s2 = 2.0 * s, hs = -0.5 * s;
    E koc[NC], kod[ND], jcd[NJ4];
#pragma unroll
    for (int k = 0; k < NC; ++k) koc[k] = 0;
#pragma unroll
    for (int l = 0; l < ND; ++l) kod[l] = 0;
#pragma unroll
    for (int v = 0; v < NJ4; ++v) jcd[v] = 0;
#pragma unroll
    for (int x = 0; x < NX; ++x) {
        issue(x + 1);
        cp_async_wait<NBUF - 1>();  // this thread's copies of slab x have landed
        const E* es = eb + (x % NBUF) * SLAB * T;
        E pxd[ND], kx[NK4], jox = 0;
#pragma unroll
        for (int l = 0; l < ND; ++l) pxd[l] = sp[(SLAB + NX * NC + x * ND + l) * QB];
#pragma unroll
        for (int v = 0; v < NK4; ++v) kx[v] = 0;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const E pxc = sp[(SLAB + x * NC + k) * QB];
#pragma unroll
            for (int l = 0; l < ND; ++l) {
                const E v = es[(k * ND + l) * T];
                jox += sp[(k * ND + l) * QB] * v;
                jcd[k * ND + l] += pox[x] * v;
                if (!jonly) {
                    koc[k] += pxd[l] * v;
                    kod[l] += pxc * v;
                    kx[k] += pod[l] * v;       // K_Xc[x][k]
                    kx[NC + l] += poc[k] * v;  // K_Xd[x][l]
                }
            }
        }
        emit(S == 0 ? Ga(O0 + g, X0 + x) : Ga(X0 + x, O0 + g), act ? s2 * (double)jox : 0.0, ua && ub, ua && ub,
             true);
        if (!jonly) {
            const int base = group_reduce_scatter<NK4>(kx, g);
            const bool shuf = uX && (uc || ud);  // warp-uniform
#pragma unroll
            for (int v = 0; v < NK4 / 4; ++v) {
                const int y = base + v;
                const bool isc = y < NC;
                emit(Ga(X0 + x, isc ? c0 + y : d0 + (y - NC)), act && y < NK ? hs * (double)kx[v] : 0.0, shuf,
                     uX && (isc ? uc : ud), y < NK);
            }
        }
    }
    cp_async_wait<0>();
    if (!jonly) {
#pragma unroll
        for (int k = 0; k < NC; ++k)
            emit(Ga(O0 + g, c0 + k), act ? hs * (double)koc[k] : 0.0, uO && uc, uO && uc, true);
#pragma unroll
        for (int l = 0; l < ND; ++l)
            emit(Ga(O0 + g, d0 + l), act ? hs * (double)kod[l] : 0.0, uO && ud, uO && ud, true);
    }
    {
        const int base = group_reduce_scatter<NJ4>(jcd, g);
#pragma unroll
        for (int v = 0; v < NJ4 / 4; ++v) {
            const int y = base + v;
            emit(Ga(c0 + y / ND, d0 + y % ND), act && y < NC * ND ? s2 * (double)jcd[v] : 0.0, uc && ud, uc && ud,
                 y < NC * ND);
        }
    }
    if (a.stats) {  // counted once per quartet, by its lane 0
        const unsigned long long nsc = act && g == 0 ? 1ull : 0ull;
        const unsigned long long npr = valid && g == 0 ? (unsigned long long)(bra.np * ket.np) : 0ull;
        warp_add_stats(a.stats, nsc, npr, a.f32 ? nsc : 0ull);
    }
}

// Diagonal builders of a staged class (quartets (ab|ab), one per pair):
// MODE 0 writes the Schwarz factor sqrt(max|e|) (fock_build_initial_diag),
// MODE 1 applies the density screen schw^2 max(D_ab, D_aa/4, D_bb/4) < thr
// (fock_build_diag.f90:20-21); both skip elements with |e| <= 1e-10 and
// scatter with the weight (bra perms)^2/8.
template <int NA, int NB, int MODE>
__global__ void __launch_bounds__(ND_THREADS) k_scatter_diag(StagedArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= staged_count(a)) return;
    const uint2 q = staged_quartet(a, t);
    const GPair pr = a.bra[q.x];
    if (MODE == 0) {
        double m = 0.0;
        for (int r = 0; r < a.nroles; ++r) m = fmax(m, a.mx[tcol(t, a.nroles) + r * TQ]);
        a.schw[q.x] = sqrt(m);
    } else {
        const double mv = fmax(a.md[pr.sa * a.nsh + pr.sb],
                               fmax(0.25 * a.md[pr.sb * a.nsh + pr.sb], 0.25 * a.md[pr.sa * a.nsh + pr.sa]));
        const double sw = a.schw[q.x];
        if (sw * sw * mv < a.thr) return;
    }
    double* e = a.out + tcol(t, NA * NB * NA * NB);
#pragma unroll 1
    for (int i = 0; i < NA * NB * NA * NB; ++i) {
        const double v = e[(size_t)i * TQ];
        if (!(fabs(v) > INTTHRESH)) e[(size_t)i * TQ] = 0.0;  // element skip
    }
    const double f = pr.sa == pr.sb ? 1.0 : 2.0;
    scatter_strided<NA, NB, NA, NB>(e, TQ, f * f / 8.0, pr, pr, a.P, a.G, a.nb, false);
}

typedef void (*NDKernel)(NDArgs);
typedef void (*DiagKernel)(DiagArgs);
typedef void (*StagedKernel)(StagedArgs);
constexpr int MAXR = 64;

// Kernels of one quartet class, filled by the class's translation unit.
// mode 0: direct (nd64/nd32); 1: staged output roles (sb*); 2: staged
// accumulator roles (sa*) then output roles (sb*).  All staged classes end
// with scat.
struct ClassKernels {
    int mode;
    NDKernel nd64, nd32;
    DiagKernel diag0, diag1;  // only for classes (X|X)
    int nd_threads, nd_qpb;   // block size and quartets per block
    int dg_threads, dg_ppb;   // block size and pairs per block (diag)
    int nacc, nrole_a, nrole_b;
    int nrole_b32;            // output roles of the FP32 chunks (staged2: larger roles)
    int nrole_a32;            // accumulator roles of the FP32 chunks (staged3: larger groups)
    StagedKernel sa64[MAXR], sa32[MAXR], sb64[MAXR], sb32[MAXR], scat;
    StagedKernel dscat0, dscat1;  // staged diagonal builders (classes (X|X))
    int scat_smem;                // dynamic shared memory of scat (bytes)
    StagedKernel scat32;          // scatter of FP32 chunks (float rows), or nullptr
    int scat32_smem;
    // grouped scatter (four lanes per quartet) where a bra shell has four
    // functions, else nullptr
    StagedKernel scatg, scatg32;
    int scatg_smem, scatg32_smem;
    int grp64, grp32;             // the grouped scatter is the default for FP64 / FP32 chunks
    // every role of a stage in one launch (gridDim.y = roles), for small chunks
    StagedKernel ma64, ma32;      // stage-A roles (staged3)
    StagedKernel mb64, mb32;      // output / HRR roles
    int bi, ki, L, nout;
};

}  // namespace hfgpu
