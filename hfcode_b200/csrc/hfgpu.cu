// B200 (sm_100a) direct-SCF Fock builder: device kernels and the C ABI.
//
// Replaces the reference's fock_build_initial_diag / fock_build_diag /
// fock_build_non_diag (+ _j_only) subroutines (brichjnh/hfcode, Fortran +
// OpenMP) with CUDA kernels that keep every piece of state resident in HBM:
//
//   k_maxdm        evaluate_maxdm.f90:1-101 -- max |P| per shell-pair block
//                  (incl. the reference's d-l block choice, evaluate_maxdm.f90:82-89)
//   k_diag<C,M>    fock_build_initial_diag.f90 (M=0: Schwarz factors, element
//                  skip |e|>1e-10) and fock_build_diag.f90 (M=1: density
//                  screen schw^2*max(D_ab,D_aa/4,D_bb/4) < thr)
//   k_screen       the per-quartet screen of fock_build_non_diag.f90:63-67
//                  (schw_ab*schw_cd*max(Dcoul,Dexch/4) < thr), evaluated for
//                  every candidate pair of active shell pairs and compacted
//                  into per-class quartet lists with warp ballots
//   k_nondiag<C>   one thread per screened shell quartet: contracted (ab|cd)
//                  from the generated class function, the post-screen
//                  max|e| < thr (fock_build_non_diag.f90:69), then the J/K
//                  scatter with FP64 atomics into a one-triangle buffer G
//   k_symm         F += G + G^T (the reference writes both triangles)
//
// The reference's per-case scatter branches (aa|aa), (aa|bc), (ab|cd), ...
// (fock_build_non_diag.f90:70-117 and 45 more blocks) all add the standard
// RHF J - K/2 contribution of each unique AO quartet; here every ordered
// component of a shell quartet carries the quartet's uniform degeneracy weight
// s = (bra perms)(ket perms)(bra-ket perms)/8, which sums to the same F.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/hfgpu.h"
#include "common.cuh"
#include "generated/class_table.inc"
#include "pairs.hpp"

namespace hfgpu {
#define HF_DECL_REG(ci) void register_class_##ci(ClassKernels* k);
HF_FOR_EACH_CLASS(HF_DECL_REG)
#undef HF_DECL_REG
static_assert(HF_NPT == NPT && HF_NCLS == NCLS, "generated class table out of date");
}  // namespace hfgpu

using namespace hfgpu;

namespace {

thread_local std::string g_err;

// CUDA forbids device-synchronising calls (cudaMalloc/cudaFree/
// cudaDeviceSynchronize/synchronous copies) in one thread while another
// thread records a stream capture.  Handles live in different threads when
// jobs are served concurrently, so captures and every such call of this
// library take this lock.
std::recursive_mutex g_dev_mu;
#define HF_DEVICE_LOCK std::lock_guard<std::recursive_mutex> dev_lock_(g_dev_mu)
}  // namespace

namespace hfgpu {
// error text for entry points in other translation units (onee.cu)
void set_last_error(const std::string& msg) { g_err = msg; }
std::recursive_mutex& device_mutex() { return g_dev_mu; }

// The library's stream-ordered memory pool on the current device, created
// on first use with no release threshold: memory a finished handle or job
// frees stays in the pool for the next one instead of going back to the
// driver at every synchronisation (which would map it again for the next
// served job).  It is released when the process exits.
cudaMemPool_t memory_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = pool;
    }
    return pools[dev];
}

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    cudaMemPool_t pool = memory_pool();
    if (!pool) return cudaMallocAsync(p, bytes, st);
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
}  // namespace hfgpu

namespace {

#define HF_CHECK(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            g_err = std::string(#call) + ": " + cudaGetErrorString(e_);                  \
            return HFGPU_ERR_CUDA;                                                       \
        }                                                                                \
    } while (0)

constexpr double SHTHRESH = 1e-11;      // molprops.f90:163
constexpr int NSTREAM = 8;              // class streams a handle creates (HFGPU_STREAMS of them used, default 4)
// bra and ket pair types of the 21 quartet classes (pair types i <= j, row by row)
__constant__ int CLS_BI[NCLS] = {HF_CLASS_BI_LIST};
__constant__ int CLS_KI[NCLS] = {HF_CLASS_KI_LIST};

// evaluate_maxdm.f90: one thread per unordered shell pair.
__global__ void k_maxdm(const int* __restrict__ shtyp, const int* __restrict__ aosh, int nsh, int nb,
                        const double* __restrict__ P, double* __restrict__ md) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long npair = (long long)nsh * (nsh + 1) / 2;
    if (t >= npair) return;
    int a = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)a * (a + 1) / 2 > t) --a;
    while ((long long)(a + 1) * (a + 2) / 2 <= t) ++a;
    const int b = (int)(t - (long long)a * (a + 1) / 2);
    auto rank = [](int ty) { return ty == 1 ? 0 : ty == 2 ? 1 : ty == 3 ? 2 : 3; };
    auto nf = [](int ty) { return ty == 1 ? 1 : ty == 2 ? 3 : ty == 3 ? 5 : 4; };
    int r = a, c = b;  // the reference's list orientation: lower rank first
    if (rank(shtyp[r]) > rank(shtyp[c])) { int x = r; r = c; c = x; }
    int nr = nf(shtyp[r]), nc = nf(shtyp[c]);
    if (shtyp[r] == 3 && shtyp[c] == 12) { nr = 4; nc = 5; }  // evaluate_maxdm.f90:82-89
    const int r0 = aosh[r], c0 = aosh[c];
    double m = 0.0;
    for (int i = 0; i < nr; ++i)
        for (int j = 0; j < nc; ++j) {
            const int row = r0 + i, col = c0 + j;
            if (row < nb && col < nb) m = fmax(m, fabs(P[row + (size_t)col * nb]));
        }
    md[(size_t)a * nsh + b] = m;
    md[(size_t)b * nsh + a] = m;
}

// One screening sub-class: the candidates of quartet class `cls` whose bra
// pairs come from one primitive-count group of the active bra list and ket
// pairs from one group of the ket list, so that every quartet in the
// compacted sub-list runs its primitive loops with the same trip counts.
struct ScreenSub {
    long long start;   // first padded candidate index
    long long ncand;   // candidates (unpadded)
    int cls;
    int same;          // one group against itself: pairs i > j only
    int b0, nbra;      // bra range in the active list
    int k0, nket;      // ket range
    long long off[2];  // write offsets of the FP64 / FP32 entries (second pass)
};

struct ScreenArgs {
    const ScreenSub* subs;
    int nsub;
    long long ntot;
    const int2* sh[NPT];      // (sa, sb) per active pair, per pair type
    const double* schw[NPT];  // Schwarz factor per active pair
    const double* md;
    int nsh;
    double thr;
    int jonly;
    double f32cut;
    unsigned long long* cnt;  // [2*nsub]: pass 1 counts, pass 2 positions
    uint2* qbuf;
};

// Per-quartet screen of fock_build_non_diag.f90:63-67 over every candidate
// pair of active shell pairs.  PASS 0 counts the survivors of each
// sub-class (FP64 and FP32 separately); PASS 1 writes them compacted at the
// offsets the host derived from those counts.  Candidates of each sub-class
// are padded to a multiple of 32 so a warp never spans two sub-classes.
template <int PASS>
__global__ void k_screen(ScreenArgs a) {
    const int lane = threadIdx.x & 31;
    const long long nwarps_total = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < a.ntot;
         w += nwarps_total) {
        const long long w0 = w * 32;
        int lo_i = 0, hi_i = a.nsub - 1;  // last sub with start <= w0
        while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i + 1) >> 1;
            if (a.subs[mid].start <= w0) lo_i = mid;
            else hi_i = mid - 1;
        }
        const int c = lo_i;
        const ScreenSub S = a.subs[c];
        const long long u = w0 + lane - S.start;
        bool pass = false, lo = false;
        unsigned ii = 0, jj = 0;
        if (u < S.ncand) {
            long long i, j;
            if (S.same) {
                i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)u)) * 0.5);
                while (i * (i - 1) / 2 > u) --i;
                while ((i + 1) * i / 2 <= u) ++i;
                j = u - i * (i - 1) / 2;
            } else {
                i = u / S.nket;
                j = u - i * S.nket;
            }
            ii = (unsigned)(S.b0 + i);
            jj = (unsigned)(S.k0 + j);
            const int bt = 0;  // pair types are resolved through the class
            (void)bt;
            const int2 ab = a.sh[CLS_BI[S.cls]][ii], cd = a.sh[CLS_KI[S.cls]][jj];
            const double dc = fmax(a.md[ab.x * a.nsh + ab.y], a.md[cd.x * a.nsh + cd.y]);
            double v = dc;
            if (!a.jonly) {
                const double dx = fmax(fmax(a.md[ab.x * a.nsh + cd.x], a.md[ab.x * a.nsh + cd.y]),
                                       fmax(a.md[ab.y * a.nsh + cd.x], a.md[ab.y * a.nsh + cd.y]));
                v = fmax(dc, 0.25 * dx);
            }
            const double bound = a.schw[CLS_BI[S.cls]][ii] * a.schw[CLS_KI[S.cls]][jj] * v;
            pass = !(bound < a.thr);
            lo = pass && bound < a.f32cut;
        }
        const unsigned m64 = __ballot_sync(0xffffffffu, pass && !lo);
        const unsigned m32 = __ballot_sync(0xffffffffu, lo);
        unsigned long long b64 = 0, b32 = 0;
        if (lane == 0) {
            if (m64) b64 = atomicAdd(&a.cnt[2 * c], (unsigned long long)__popc(m64));
            if (m32) b32 = atomicAdd(&a.cnt[2 * c + 1], (unsigned long long)__popc(m32));
        }
        if (PASS == 1) {
            b64 = __shfl_sync(0xffffffffu, b64, 0);
            b32 = __shfl_sync(0xffffffffu, b32, 0);
            const unsigned lt = (1u << lane) - 1u;
            if (pass && !lo) a.qbuf[S.off[0] + (long long)b64 + __popc(m64 & lt)] = make_uint2(ii, jj);
            if (lo) a.qbuf[S.off[1] + (long long)b32 + __popc(m32 & lt)] = make_uint2(ii, jj);
        }
    }
}

// Sub-class ranges and list regions of the classes (fixed after the Schwarz
// pass), passed by value to k_offsets.
struct OffsetArgs {
    int csub[NCLS + 1];      // sub-classes of class c: [csub[c], csub[c+1])
    long long coff[NCLS];    // first entry of class c in the quartet buffer
};

// Write offsets of the compacted lists from the pass-0 counts, on the device
// so that a build needs no host round trip: per class its FP64 entries, then
// its FP32 entries, sub-classes in order.  Also stores the per-class totals
// that the class kernels read.  One thread per class.
__global__ void k_offsets(OffsetArgs o, ScreenSub* __restrict__ subs, const unsigned long long* __restrict__ cnt,
                          unsigned long long* __restrict__ ncls) {
    const int c = threadIdx.x;
    if (c >= NCLS) return;
    unsigned long long n64 = 0, n32 = 0;
    for (int k = o.csub[c]; k < o.csub[c + 1]; ++k) {
        n64 += cnt[2 * k];
        n32 += cnt[2 * k + 1];
    }
    long long p64 = o.coff[c], p32 = o.coff[c] + (long long)n64;
    for (int k = o.csub[c]; k < o.csub[c + 1]; ++k) {
        subs[k].off[0] = p64;
        subs[k].off[1] = p32;
        p64 += (long long)cnt[2 * k];
        p32 += (long long)cnt[2 * k + 1];
    }
    ncls[2 * c] = n64;
    ncls[2 * c + 1] = n32;
}

// The density in shell-pair blocks: block (s1, s2) holds P[r][c] for the
// functions r of shell s1 and c of shell s2, row-major, at boff[s1*nsh+s2].
// Rows the scatter reads become contiguous (one element per column before).
__global__ void k_pblock(const double* __restrict__ P, double* __restrict__ Pb, const int2* __restrict__ aomap,
                         const int* __restrict__ nfsh, const int* __restrict__ boff, int nb, int nsh) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nb * nb) return;
    const int r = (int)(t % nb), c = (int)(t / nb);
    const int2 mr = aomap[r], mc = aomap[c];  // (shell, function within the shell)
    Pb[boff[mr.x * nsh + mc.x] + mr.y * nfsh[mc.x] + mc.y] = P[t];
}

// FMA-chain throughput probe: 8 independent chains per thread so the FP64 and
// FP32 pipes, not latency, bound it.  Used to state the FP64/FP32 roofline.
template <typename T>
__global__ void k_fma_peak(T* out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (T)(threadIdx.x + i);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = x[i] * a + b;
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == (T)-1.2345) out[0] = s;  // keeps the chains live
}

__global__ void k_symm(double* __restrict__ F, const double* __restrict__ G, int nb) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nb * nb) return;
    const int i = (int)(t % nb), j = (int)(t / nb);
    F[t] += G[t] + G[j + (size_t)i * nb];
}

// ------------------------------------------------------------- host ----
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
};

}  // namespace

struct hfgpu_handle {
    int nsh = 0, nb = 0, npairs = 0;
    std::vector<int> shtyp, nzet, aosh;
    std::vector<HostPair> pairs[NPT];     // all pairs per GPU type
    std::vector<int> refcount;            // pairs per reference class
    std::vector<double> schw[NPT];        // host copy, by pair index
    std::vector<int> last_ref;            // lastXX per reference class
    bool have_schwarz = false;
    int timing = 0;
    int device = 0;                       // the CUDA device current at hfgpu_init
    long long merge_blocks = 0;           // chunks up to this many role blocks run one launch per stage
    int grouped_scatter = 1;              // four-lane scatter: 1 per class tuning, 2 everywhere, 0 nowhere
    int nstreams = 4;                     // class streams the off-diagonal build uses (<= NSTREAM)
    cudaStream_t stream = nullptr;
    cudaStream_t aux[NSTREAM] = {};    // independent classes run concurrently on these
    cudaEvent_t fork = nullptr, join[NSTREAM] = {};
    // device
    int* d_shtyp = nullptr;
    int* d_aosh = nullptr;
    double* d_psoa = nullptr;      // all-pairs primitive arrays (SoA)
    PrimSoA psoa{};
    double* d_apsoa = nullptr;     // active lists' interleaved primitive arrays (SoA)
    PrimSoA apsoa{};
    std::vector<GPrim> hprims;     // host copy, all-pairs order
    GPair* d_pairs[NPT] = {};
    double* d_schw[NPT] = {};
    GPair* d_apairs[NPT] = {};
    int2* d_ash[NPT] = {};
    double* d_aschw[NPT] = {};
    int nact[NPT] = {};
    std::vector<int> act_np[NPT];
    double* d_boys = nullptr;
    float* d_boysf = nullptr;
    double* d_P = nullptr;
    double* d_F = nullptr;
    double* d_G = nullptr;
    double* d_md = nullptr;
    ScreenSub* d_subs = nullptr;
    std::vector<ScreenSub> hsubs;
    size_t subcap = 0;
    uint2* d_q = nullptr;
    size_t qcap = 0;
    double* d_scratch = nullptr;   // staged classes: accumulators, outputs, maxima
    uint2* d_diaglist[NPT] = {};   // (i, i) for every pair of a type: staged diagonal builders
    double* d_dscratch = nullptr;  // scratch of the staged diagonal builders
    size_t dstride[NPT] = {};
    size_t scratch_doubles = 0;
    size_t dscratch_doubles = 0;   // scratch of the staged diagonal builders
    size_t stride[NCLS] = {};      // quartets per chunk of each staged class
    size_t slot_doubles = 0;       // scratch per class stream
    size_t scratch_budget = 0;     // bytes; 0 = default (HFGPU_SCRATCH_MB, or 24 GiB capped at device memory / 6)
    size_t naprims = 0;            // primitive pairs of the active lists
    unsigned long long* d_cnt = nullptr;
    ClassStats* d_stats = nullptr;
    // last build statistics
    double st_ms[NCLS] = {};
    long long ntot = 0;
    long long ccap[NCLS] = {};      // candidates per class (upper bound of its list)
    long long coff[NCLS] = {};      // class region in the quartet buffer
    long long n64[NCLS] = {}, n32[NCLS] = {};
    cudaEvent_t ev[2 * NCLS + 2] = {};
    int nsm = 148;
    long long launches = 0;             // kernels enqueued by this handle (graph replays included)
    long long graph_launches = 0;       // kernels in the captured build
    OffsetArgs offs{};                  // sub-class ranges / list regions per class
    unsigned long long* d_ncls = nullptr;  // [2 * NCLS] surviving quartets (FP64, FP32) per class
    double* d_Pb = nullptr;             // density in shell-pair blocks (nb x nb)
    int* d_boff = nullptr;              // block offsets (nsh x nsh)
    int2* d_aomap = nullptr;            // per function: (shell, index within the shell)
    int* d_nfsh = nullptr;              // functions per shell
    cudaGraph_t graph = nullptr;        // captured full build (hfgpu_graph_capture)
    cudaGraphExec_t gexec = nullptr;
    const void* gkey_f = nullptr;       // what the capture was recorded with
    const void* gkey_p = nullptr;
    double gkey_thr[3] = {};
};

struct hfgpu_batch {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<hfgpu_handle*> hs;  // launch accounting
};

namespace {

int set_err(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

// Device buffers of a handle come from the library's stream-ordered pool on
// the handle's stream: cudaFreeAsync, unlike cudaFree, does not synchronise
// the whole device, so a served job that finishes does not stall the jobs
// still running on the GPU.  These calls need no lock: a capture in another
// thread (thread-local mode) is unaffected by them.
template <typename T>
int dalloc(T** p, size_t n, cudaStream_t st) {
    if (n == 0) n = 1;
    cudaError_t e = pool_alloc((void**)p, n * sizeof(T), st);
    if (e != cudaSuccess) {
        *p = nullptr;
        g_err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return HFGPU_ERR_NOMEM;
    }
    return HFGPU_OK;
}

template <typename T>
void dfree(T*& p, cudaStream_t st) {
    if (p) cudaFreeAsync((void*)p, st);
    p = nullptr;
}

// class index of pair types (i <= j) in the generator's class order
int class_index(int i, int j) {
    static const int bi[NCLS] = {HF_CLASS_BI_LIST}, ki[NCLS] = {HF_CLASS_KI_LIST};
    for (int c = 0; c < NCLS; ++c)
        if (bi[c] == i && ki[c] == j) return c;
    return -1;
}

struct ClassTable {
    ClassKernels k[NCLS]{};
    ClassTable() {
#define HF_REG_PTR(ci) register_class_##ci,
        void (*reg[NCLS])(ClassKernels*) = {HF_FOR_EACH_CLASS(HF_REG_PTR)};
#undef HF_REG_PTR
        for (int c = 0; c < NCLS; ++c) {
            reg[c](&k[c]);
            // the staged scatter streams its rows through > 48 KB of shared memory
            if (k[c].scat && k[c].scat_smem > 0)
                cudaFuncSetAttribute(k[c].scat, cudaFuncAttributeMaxDynamicSharedMemorySize, k[c].scat_smem);
            if (k[c].scat32 && k[c].scat32_smem > 0)
                cudaFuncSetAttribute(k[c].scat32, cudaFuncAttributeMaxDynamicSharedMemorySize, k[c].scat32_smem);
            if (k[c].scatg && k[c].scatg_smem > 0)
                cudaFuncSetAttribute(k[c].scatg, cudaFuncAttributeMaxDynamicSharedMemorySize, k[c].scatg_smem);
            if (k[c].scatg32 && k[c].scatg32_smem > 0)
                cudaFuncSetAttribute(k[c].scatg32, cudaFuncAttributeMaxDynamicSharedMemorySize, k[c].scatg32_smem);
            // The role kernels use no shared memory: they prefer the largest
            // L1 carve-out (HFGPU_CARVEOUT=<percent of shared memory> or
            // "none" overrides).  With the four class streams, where role and
            // scatter kernels of different classes share SMs, the C60 FP64
            // build measured 207.6 ms without the preference and 198.4 ms with
            // it; the class times alone are unchanged.  The same preference on
            // the scatters (shared memory first) or on the direct kernels (L1
            // first) measured slower (205.0 and 202.6 ms).
            int pct = 0;
            if (const char* e = getenv("HFGPU_CARVEOUT")) pct = strcmp(e, "none") == 0 ? -2 : atoi(e);
            auto pref = [](StagedKernel f, int v) {
                if (f && v >= -1) cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, v);
            };
            for (int r = 0; r < MAXR; ++r) {
                pref(k[c].sa64[r], pct);
                pref(k[c].sa32[r], pct);
                pref(k[c].sb64[r], pct);
                pref(k[c].sb32[r], pct);
            }
            pref(k[c].ma64, pct);
            pref(k[c].ma32, pct);
            pref(k[c].mb64, pct);
            pref(k[c].mb32, pct);
        }
    }
};
const ClassTable& class_table() {
    static ClassTable t;
    return t;
}
#define CLASS_KERNELS (class_table().k)

DiagKernel diag_kernel(int pt, int mode) {
    const ClassKernels& k = CLASS_KERNELS[class_index(pt, pt)];
    return mode ? k.diag1 : k.diag0;
}

size_t scratch_budget_doubles();

int upload_fp(hfgpu_handle* h, const double* f, const double* p) {
    size_t bytes = (size_t)h->nb * h->nb * sizeof(double);
    HF_CHECK(cudaMemcpyAsync(h->d_P, p, bytes, cudaMemcpyHostToDevice, h->stream));
    HF_CHECK(cudaMemcpyAsync(h->d_F, f, bytes, cudaMemcpyHostToDevice, h->stream));
    return HFGPU_OK;
}

int download_f(hfgpu_handle* h, double* f) {
    size_t bytes = (size_t)h->nb * h->nb * sizeof(double);
    HF_CHECK(cudaMemcpyAsync(f, h->d_F, bytes, cudaMemcpyDeviceToHost, h->stream));
    HF_CHECK(cudaStreamSynchronize(h->stream));
    return HFGPU_OK;
}

int launch_maxdm(hfgpu_handle* h, const double* P, double* md = nullptr) {
    long long np = (long long)h->nsh * (h->nsh + 1) / 2;
    int blocks = (int)((np + 255) / 256);
    ++h->launches;
    k_maxdm<<<blocks, 256, 0, h->stream>>>(h->d_shtyp, h->d_aosh, h->nsh, h->nb, P, md ? md : h->d_md);
    HF_CHECK(cudaGetLastError());
    return HFGPU_OK;
}

int launch_symm(hfgpu_handle* h, double* F, const double* G = nullptr) {
    long long n = (long long)h->nb * h->nb;
    ++h->launches;
    k_symm<<<(int)((n + 255) / 256), 256, 0, h->stream>>>(F, G ? G : h->d_G, h->nb);
    HF_CHECK(cudaGetLastError());
    return HFGPU_OK;
}

// Whether a chunk runs every role of a stage in one launch (gridDim.y =
// roles): when all its role blocks together are at most the handle's
// merge_blocks (eight per SM).  Large chunks keep one launch per role, so that every warp on an SM
// runs the same role's code (these FP64 recursions are long straight-line
// programs, and an SM running several of them thrashes its instruction
// cache); small chunks gain more from filling the SMs and launching less.
bool merge_roles(const hfgpu_handle* h, const ClassKernels& K, int blocks, int roles) {
    return K.mb64 && roles > 1 && (long long)blocks * roles <= h->merge_blocks;
}

// Diagonal builder of a staged pair type: chunks of its pairs through the
// class's roles and k_scatter_diag.
int run_staged_diag(hfgpu_handle* h, int t, int mode, const double* P, double thr, double* G, const double* md) {
    const ClassKernels& K = CLASS_KERNELS[class_index(t, t)];
    const long long n = (long long)h->pairs[t].size();
    const size_t st = h->dstride[t];
    for (long long q0 = 0; q0 < n; q0 += (long long)st) {
        const int m = (int)std::min<long long>((long long)st, n - q0);
        StagedArgs a{};
        a.quartets = h->d_diaglist[t];
        a.n = m;
        a.q0 = q0;
        a.ncls = nullptr;
        a.bra = h->d_pairs[t];
        a.ket = h->d_pairs[t];
        a.prims = h->psoa;
        a.boys = h->d_boys;
        a.boysf = h->d_boysf;
        a.acc = h->d_dscratch;
        a.out = h->d_dscratch + (size_t)K.nacc * st;
        a.mx = h->d_dscratch + (size_t)(K.nacc + K.nout) * st;
        a.stride = st;
        a.nroles = K.nrole_b;
        a.P = P;
        a.G = G;
        a.nb = h->nb;
        a.thr = thr;
        a.stats = nullptr;
        a.schw = h->d_schw[t];
        a.md = md;
        a.nsh = h->nsh;
        const int blocks = (m + ND_THREADS - 1) / ND_THREADS;
        if (merge_roles(h, K, blocks, std::max(K.nrole_a, K.nrole_b))) {
            if (K.nrole_a > 0) {
                ++h->launches;
                K.ma64<<<dim3(blocks * RB_SCALE, K.nrole_a), RB_THREADS, 0, h->stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
            ++h->launches;
            K.mb64<<<dim3(blocks * RB_SCALE, K.nrole_b), RB_THREADS, 0, h->stream>>>(a);
            HF_CHECK(cudaGetLastError());
        } else {
            for (int r = 0; r < K.nrole_a; ++r) {
                ++h->launches;
                K.sa64[r]<<<blocks * RB_SCALE, RB_THREADS, 0, h->stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
            for (int r = 0; r < K.nrole_b; ++r) {
                ++h->launches;
                K.sb64[r]<<<blocks * RB_SCALE, RB_THREADS, 0, h->stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
        }
        ++h->launches;
        (mode ? K.dscat1 : K.dscat0)<<<blocks, ND_THREADS, 0, h->stream>>>(a);
        HF_CHECK(cudaGetLastError());
    }
    return HFGPU_OK;
}

int launch_diag(hfgpu_handle* h, int mode, const double* P, double thr, double* G = nullptr,
                const double* md = nullptr) {
    for (int t = 0; t < NPT; ++t) {
        int n = (int)h->pairs[t].size();
        if (n == 0) continue;
        if (CLASS_KERNELS[class_index(t, t)].mode != 0) {
            int rc = run_staged_diag(h, t, mode, P, thr, G ? G : h->d_G, md ? md : h->d_md);
            if (rc) return rc;
            continue;
        }
        DiagArgs a{h->d_pairs[t], n, h->psoa, h->d_boys, h->d_schw[t], md ? md : h->d_md, h->nsh, P,
                   G ? G : h->d_G, h->nb, thr};
        const ClassKernels& K = CLASS_KERNELS[class_index(t, t)];
        ++h->launches;
        diag_kernel(t, mode)<<<(n + K.dg_ppb - 1) / K.dg_ppb, K.dg_threads, 0, h->stream>>>(a);
        HF_CHECK(cudaGetLastError());
    }
    return HFGPU_OK;
}

// Default scratch budget: 24 GiB, at most a sixth of the device's memory.
// Larger chunks mean fewer role/scatter launches per class and shorter
// tails: C60 builds 226.3 ms at 6 GiB, 220.5 ms at 24 GiB.  A handle
// allocates only what its largest class list needs (the chunk stride is
// capped by the class capacity), so small molecules take far less.
size_t scratch_budget_doubles() {
    size_t mb = 24576;
    size_t freeb = 0, totalb = 0;
    if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess && totalb > 0)
        mb = std::min(mb, totalb / 6 / (1024 * 1024));
    if (const char* e = getenv("HFGPU_SCRATCH_MB")) {
        long v = atol(e);
        if (v > 0) mb = (size_t)v;
    }
    return mb * 1024 * 1024 / sizeof(double);
}

// Schwarz ordering (index_sort + find_threshold) and the active pair arrays.
int build_active(hfgpu_handle* h) {
    // no library lock here: the allocations are stream-ordered, and holding
    // the lock across this function's stream synchronisations made the jobs
    // of a server queue behind one another's GPU work
    for (int t = 0; t < NPT; ++t) {
        int n = (int)h->pairs[t].size();
        h->schw[t].resize(n);
        if (n)
            HF_CHECK(cudaMemcpyAsync(h->schw[t].data(), h->d_schw[t], n * sizeof(double), cudaMemcpyDeviceToHost,
                                     h->stream));
    }
    HF_CHECK(cudaStreamSynchronize(h->stream));
    h->last_ref.assign(10, 0);
    long long total_q = 0;
    std::vector<GPrim> aprims;
    std::vector<GPair> aps[NPT];
    std::vector<int2> ashs[NPT];
    std::vector<double> ascs[NPT];
    for (int t = 0; t < NPT; ++t) {
        const int n = (int)h->pairs[t].size();
        // reference list order is refpos; pairs[t] is stored in that order
        std::vector<int> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return h->schw[t][x] > h->schw[t][y]; });
        int last = 0;
        if (n > 0) {
            if (h->schw[t][ord[0]] < SHTHRESH) last = 1;
            else if (h->schw[t][ord[n - 1]] > SHTHRESH) last = n;
            else {
                last = n;
                for (int i = 0; i < n; ++i)
                    if (h->schw[t][ord[i]] < SHTHRESH) { last = i + 1; break; }
            }
        }
        h->last_ref[GPU_TO_REF[t]] = last;
        // active set, re-ordered for the GPU: primitive count, first shell, then Schwarz
        std::vector<int> act(ord.begin(), ord.begin() + last);
        std::stable_sort(act.begin(), act.end(), [&](int x, int y) {
            int nx = h->pairs[t][x].g.np, ny = h->pairs[t][y].g.np;
            if (nx != ny) return nx > ny;
            // within a primitive-count group by first shell, so the 32
            // quartets of a warp mostly share it (the staged scatter then
            // adds their K blocks with one atomic per element)
            const int sx = h->pairs[t][x].g.sa, sy = h->pairs[t][y].g.sa;
            if (sx != sy) return sx < sy;
            return h->schw[t][x] > h->schw[t][y];
        });
        std::vector<GPair> ap(last);
        std::vector<int2> ash(last);
        std::vector<double> asc(last);
        for (int i = 0; i < last; ++i) {
            ap[i] = h->pairs[t][act[i]].g;
            ash[i] = make_int2(ap[i].sa, ap[i].sb);
            asc[i] = h->schw[t][act[i]];
        }
        h->nact[t] = last;
        h->act_np[t].resize(last);
        for (int i = 0; i < last; ++i) h->act_np[t][i] = ap[i].np;
        // interleave the primitives of equal-count neighbours: entry ik of
        // pair i of a group [g0, g0+ng) goes to base + ik*ng + (i - g0)
        for (int i = 0; i < last;) {
            int j = i + 1;
            while (j < last && ap[j].np == ap[i].np) ++j;
            const int ng = j - i, np = ap[i].np;
            const size_t base = aprims.size();
            aprims.resize(base + (size_t)np * ng);
            for (int k = i; k < j; ++k) {
                for (int ik = 0; ik < np; ++ik) aprims[base + (size_t)ik * ng + (k - i)] = h->hprims[ap[k].p0 + ik];
                ap[k].p0 = (int)(base + (k - i));
                ap[k].ps = ng;
            }
            i = j;
        }
        aps[t] = std::move(ap);
        ashs[t] = std::move(ash);
        ascs[t] = std::move(asc);
    }
    {
        std::vector<double> soa = prims_soa(aprims);
        dfree(h->d_apsoa, h->stream);
        int rc = dalloc(&h->d_apsoa, std::max<size_t>(soa.size(), 1), h->stream);
        if (rc) return rc;
        h->apsoa = soa_view(h->d_apsoa, aprims.size());
        h->naprims = aprims.size();
        if (!soa.empty())
            HF_CHECK(cudaMemcpyAsync(h->d_apsoa, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice,
                                     h->stream));
        for (int t = 0; t < NPT; ++t) {
            const int last = h->nact[t];
            if (!last) continue;
            HF_CHECK(cudaMemcpyAsync(h->d_apairs[t], aps[t].data(), last * sizeof(GPair), cudaMemcpyHostToDevice,
                                     h->stream));
            HF_CHECK(cudaMemcpyAsync(h->d_ash[t], ashs[t].data(), last * sizeof(int2), cudaMemcpyHostToDevice,
                                     h->stream));
            HF_CHECK(cudaMemcpyAsync(h->d_aschw[t], ascs[t].data(), last * sizeof(double), cudaMemcpyHostToDevice,
                                     h->stream));
        }
        HF_CHECK(cudaStreamSynchronize(h->stream));
    }
    // screening sub-classes: primitive-count groups of the active lists
    std::vector<std::pair<int, int>> groups[NPT];  // (start, length)
    for (int t = 0; t < NPT; ++t) {
        const int n = h->nact[t];
        for (int i = 0; i < n;) {
            int j = i + 1;
            while (j < n && h->act_np[t][j] == h->act_np[t][i]) ++j;
            groups[t].push_back({i, j - i});
            i = j;
        }
    }
    h->hsubs.clear();
    long long start = 0, qoff = 0;
    for (int c = 0; c < NCLS; ++c) {
        const int bi = CLASS_KERNELS[c].bi, ki = CLASS_KERNELS[c].ki;
        long long ccap = 0;
        for (size_t gb = 0; gb < groups[bi].size(); ++gb)
            for (size_t gk = 0; gk < groups[ki].size(); ++gk) {
                if (bi == ki && gk > gb) continue;  // pairs (ii, jj) with ii > jj only
                ScreenSub sub{};
                sub.cls = c;
                sub.same = (bi == ki && gb == gk);
                sub.b0 = groups[bi][gb].first;
                sub.nbra = groups[bi][gb].second;
                sub.k0 = groups[ki][gk].first;
                sub.nket = groups[ki][gk].second;
                sub.ncand = sub.same ? (long long)sub.nbra * (sub.nbra - 1) / 2 : (long long)sub.nbra * sub.nket;
                if (sub.ncand == 0) continue;
                sub.start = start;
                start += (sub.ncand + 31) / 32 * 32;
                ccap += sub.ncand;
                h->hsubs.push_back(sub);
            }
        h->ccap[c] = ccap;
        h->coff[c] = qoff;
        h->offs.coff[c] = qoff;
        qoff += ccap;
        h->offs.csub[c + 1] = (int)h->hsubs.size();
    }
    h->offs.csub[0] = 0;
    h->ntot = start;
    total_q = qoff;
    if (h->hsubs.size() > h->subcap) {
        dfree(h->d_subs, h->stream);
        h->subcap = 0;
        int rc = dalloc(&h->d_subs, h->hsubs.size(), h->stream);
        if (rc) return rc;
        dfree(h->d_cnt, h->stream);
        rc = dalloc(&h->d_cnt, 2 * h->hsubs.size(), h->stream);
        if (rc) return rc;
        h->subcap = h->hsubs.size();
    }
    // the sub-class table stays on the device; k_offsets fills its offsets
    if (!h->hsubs.empty()) {
        HF_CHECK(cudaMemcpyAsync(h->d_subs, h->hsubs.data(), h->hsubs.size() * sizeof(ScreenSub),
                                 cudaMemcpyHostToDevice, h->stream));
        HF_CHECK(cudaStreamSynchronize(h->stream));
    }
    if ((size_t)total_q > h->qcap) {
        dfree(h->d_q, h->stream);
        h->qcap = 0;
        int rc = dalloc(&h->d_q, (size_t)total_q, h->stream);
        if (rc) return rc;
        h->qcap = (size_t)std::max<long long>(total_q, 1);
    }
    // scratch of the staged classes: one chunk of stride quartets holds
    // (accumulators + outputs + role maxima) doubles per quartet
    size_t need = 0;
    const size_t budget = (h->scratch_budget ? h->scratch_budget / sizeof(double) : scratch_budget_doubles()) /
                          h->nstreams;  // one slot per class stream
    for (int c = 0; c < NCLS; ++c) {
        const ClassKernels& K = CLASS_KERNELS[c];
        h->stride[c] = 0;
        if (K.mode == 0 || h->ccap[c] == 0) continue;
        const size_t per = (size_t)K.nacc + K.nout + std::max(K.nrole_b, K.nrole_b32);
        size_t st = std::min<size_t>((size_t)h->ccap[c], budget / per);
        st = (std::max<size_t>(st, TQ) + TQ - 1) / TQ * TQ;  // whole scratch tiles
        h->stride[c] = st;
        need = std::max(need, st * per);
    }
    if (need * h->nstreams > h->scratch_doubles) {
        dfree(h->d_scratch, h->stream);
        h->scratch_doubles = 0;
        int rc = dalloc(&h->d_scratch, need * h->nstreams, h->stream);
        if (rc) return rc;
        h->scratch_doubles = need * h->nstreams;
    }
    h->slot_doubles = need;
    h->have_schwarz = true;
    return HFGPU_OK;
}

// Staged class: chunks of the quartet list through the accumulator roles
// (mode 2), the output roles and the scatter kernel.
int run_staged(hfgpu_handle* h, int c, int prec, long long n, const double* P, double thr, int jonly,
               cudaStream_t stream, double* scratch) {
    const ClassKernels& K = CLASS_KERNELS[c];
    const size_t st = h->stride[c];
    for (long long q0 = 0; q0 < n; q0 += (long long)st) {
        const int m = (int)std::min<long long>((long long)st, n - q0);
        StagedArgs a{};
        a.quartets = h->d_q + h->coff[c];
        a.n = m;  // the kernels clamp it by the device-side count
        a.q0 = q0;
        a.ncls = h->d_ncls;
        a.cls = c;
        a.prec = prec;
        a.bra = h->d_apairs[K.bi];
        a.ket = h->d_apairs[K.ki];
        a.prims = h->apsoa;
        a.boys = h->d_boys;
        a.boysf = h->d_boysf;
        a.acc = scratch;
        a.out = scratch + (size_t)K.nacc * st;
        a.mx = scratch + (size_t)(K.nacc + K.nout) * st;
        a.stride = st;
        a.nroles = prec ? K.nrole_b32 : K.nrole_b;
        a.P = P;
        a.Pb = h->d_Pb;
        a.boff = h->d_boff;
        a.nsh = h->nsh;
        a.G = h->d_G;
        a.nb = h->nb;
        a.thr = thr;
        a.jonly = jonly;
        a.f32 = prec;
        a.stats = h->d_stats + c;
        const int blocks = (m + ND_THREADS - 1) / ND_THREADS;
        const int na = prec ? K.nrole_a32 : K.nrole_a;
        if (merge_roles(h, K, blocks, std::max(na, a.nroles))) {
            // a small chunk: every role of a stage in one launch, side by side
            if (na > 0) {
                ++h->launches;
                (prec ? K.ma32 : K.ma64)<<<dim3(blocks * RB_SCALE, na), RB_THREADS, 0, stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
            ++h->launches;
            (prec ? K.mb32 : K.mb64)<<<dim3(blocks * RB_SCALE, a.nroles), RB_THREADS, 0, stream>>>(a);
            HF_CHECK(cudaGetLastError());
        } else {
            for (int r = 0; r < na; ++r) {
                ++h->launches;
                (prec ? K.sa32[r] : K.sa64[r])<<<blocks * RB_SCALE, RB_THREADS, 0, stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
            for (int r = 0; r < a.nroles; ++r) {
                ++h->launches;
                (prec ? K.sb32[r] : K.sb64[r])<<<blocks * RB_SCALE, RB_THREADS, 0, stream>>>(a);
                HF_CHECK(cudaGetLastError());
            }
        }
        ++h->launches;
        // grouped scatter: where the class's tuning chooses it (grouped_scatter 1),
        // everywhere it exists (2) or nowhere (0)
        const bool grp = h->grouped_scatter == 2 || (h->grouped_scatter == 1 && (prec ? K.grp32 : K.grp64));
        const StagedKernel sg = grp ? (prec ? K.scatg32 : K.scatg) : nullptr;
        if (sg) {  // four lanes per quartet
            const int gblocks = (int)(((long long)m * SG + ND_THREADS - 1) / ND_THREADS);
            sg<<<gblocks, ND_THREADS, prec ? K.scatg32_smem : K.scatg_smem, stream>>>(a);
        } else if (prec && K.scat32) {
            K.scat32<<<blocks, ND_THREADS, K.scat32_smem, stream>>>(a);  // float rows
        } else {
            K.scat<<<blocks, ND_THREADS, K.scat_smem, stream>>>(a);
        }
        HF_CHECK(cudaGetLastError());
    }
    return HFGPU_OK;
}

// Off-diagonal build: the two screening passes with device-side offsets,
// then the class kernels on the handle's concurrent class streams.  With capture set,
// nothing is read back on the host: every launch is sized by the class's
// candidate count (an upper bound) and the kernels read the surviving count
// from d_ncls, so the whole sequence can be recorded into a CUDA graph.
// Eager builds read the counts back once to size the launches exactly.
int run_non_diag(hfgpu_handle* h, const double* P, double thr, int jonly, double f32cut, bool capture = false) {
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    HF_CHECK(cudaMemsetAsync(h->d_stats, 0, NCLS * sizeof(ClassStats), h->stream));
    HF_CHECK(cudaMemsetAsync(h->d_ncls, 0, 2 * NCLS * sizeof(unsigned long long), h->stream));
    const int nsub = (int)h->hsubs.size();
    for (int c = 0; c < NCLS; ++c) h->n64[c] = h->n32[c] = 0;
    if (h->ntot > 0 && nsub > 0) {
        ScreenArgs sa{};
        sa.subs = h->d_subs;
        sa.nsub = nsub;
        sa.ntot = h->ntot;
        for (int t = 0; t < NPT; ++t) {
            sa.sh[t] = h->d_ash[t];
            sa.schw[t] = h->d_aschw[t];
        }
        sa.md = h->d_md;
        sa.nsh = h->nsh;
        sa.thr = thr;
        sa.jonly = jonly;
        sa.f32cut = f32cut;
        sa.cnt = h->d_cnt;
        sa.qbuf = h->d_q;
        const long long warps = h->ntot / 32;
        const int blocks = (int)std::min<long long>((warps + 7) / 8, (long long)h->nsm * 64);
        const size_t cbytes = 2 * (size_t)nsub * sizeof(unsigned long long);
        HF_CHECK(cudaMemsetAsync(h->d_cnt, 0, cbytes, h->stream));
        ++h->launches;
        k_screen<0><<<blocks, 256, 0, h->stream>>>(sa);  // survivors per sub-class
        HF_CHECK(cudaGetLastError());
        ++h->launches;
        k_offsets<<<1, (NCLS + 31) / 32 * 32, 0, h->stream>>>(h->offs, h->d_subs, h->d_cnt, h->d_ncls);
        HF_CHECK(cudaGetLastError());
        HF_CHECK(cudaMemsetAsync(h->d_cnt, 0, cbytes, h->stream));
        ++h->launches;
        k_screen<1><<<blocks, 256, 0, h->stream>>>(sa);  // compacted write
        HF_CHECK(cudaGetLastError());
    }
    {  // the density in shell-pair blocks for the staged scatter
        const long long n = (long long)h->nb * h->nb;
        ++h->launches;
        k_pblock<<<(int)((n + 255) / 256), 256, 0, h->stream>>>(P, h->d_Pb, h->d_aomap, h->d_nfsh, h->d_boff, h->nb,
                                                                h->nsh);
        HF_CHECK(cudaGetLastError());
    }
    if (!capture) {
        unsigned long long cnt[2 * NCLS];
        HF_CHECK(cudaMemcpyAsync(cnt, h->d_ncls, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
        HF_CHECK(cudaStreamSynchronize(h->stream));
        for (int c = 0; c < NCLS; ++c) {
            h->n64[c] = (long long)cnt[2 * c];
            h->n32[c] = (long long)cnt[2 * c + 1];
        }
    }
    // work items (class, precision) over the class streams, largest
    // first onto the least-loaded stream; with timing on, everything runs in
    // order on the handle's stream
    struct Item { int c, prec; long long n; double w; };
    std::vector<Item> items;
    for (int c = 0; c < NCLS; ++c) {
        h->st_ms[c] = 0.0;
        for (int prec = 0; prec < 2; ++prec) {
            long long n = prec ? h->n32[c] : h->n64[c];
            if (capture) n = (prec && !(f32cut > 0.0)) ? 0 : h->ccap[c];
            if (n > 0) items.push_back({c, prec, n, (double)n * CLASS_KERNELS[c].nout});
        }
    }
    const bool multi = capture || !h->timing;
    if (multi) {
        std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.w > y.w; });
        HF_CHECK(cudaEventRecord(h->fork, h->stream));
        for (int k = 0; k < h->nstreams; ++k) HF_CHECK(cudaStreamWaitEvent(h->aux[k], h->fork, 0));
    }
    double load[NSTREAM] = {};
    for (const Item& it : items) {
        const int c = it.c, prec = it.prec;
        const long long n = it.n;
        const ClassKernels& K = CLASS_KERNELS[c];
        int k = 0;
        for (int q = 1; q < h->nstreams; ++q)
            if (load[q] < load[k]) k = q;
        load[k] += it.w;
        cudaStream_t st = multi ? h->aux[k] : h->stream;
        double* slot = h->d_scratch ? h->d_scratch + (multi ? (size_t)k * h->slot_doubles : 0) : nullptr;
        const bool timed = h->timing && !multi;
        if (timed) HF_CHECK(cudaEventRecord(h->ev[2 * c], h->stream));
        if (K.mode == 0) {
            NDArgs a{};
            a.quartets = h->d_q + h->coff[c];
            a.n = (int)n;
            a.ncls = h->d_ncls;
            a.cls = c;
            a.prec = prec;
            a.bra = h->d_apairs[K.bi];
            a.ket = h->d_apairs[K.ki];
            a.prims = h->apsoa;
            a.boys = h->d_boys;
            a.boysf = h->d_boysf;
            a.P = P;
            a.G = h->d_G;
            a.nb = h->nb;
            a.thr = thr;
            a.jonly = jonly;
            a.stats = h->d_stats + c;
            long long blocks = (n + K.nd_qpb - 1) / K.nd_qpb;
            if (capture) blocks = std::min<long long>(blocks, (long long)h->nsm * 16);  // grid-stride
            ++h->launches;
            (prec ? K.nd32 : K.nd64)<<<(int)blocks, K.nd_threads, 0, st>>>(a);
            HF_CHECK(cudaGetLastError());
        } else {
            int rc = run_staged(h, c, prec, n, P, thr, jonly, st, slot);
            if (rc) return rc;
        }
        if (timed) {
            HF_CHECK(cudaEventRecord(h->ev[2 * c + 1], h->stream));
            HF_CHECK(cudaEventSynchronize(h->ev[2 * c + 1]));
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev[2 * c], h->ev[2 * c + 1]);
            h->st_ms[c] += ms;
        }
    }
    if (multi) {
        for (int k = 0; k < h->nstreams; ++k) {
            HF_CHECK(cudaEventRecord(h->join[k], h->aux[k]));
            HF_CHECK(cudaStreamWaitEvent(h->stream, h->join[k], 0));
        }
    }
    return HFGPU_OK;
}

}  // namespace

extern "C" {

const char* hfgpu_last_error(void) { return g_err.c_str(); }

int hfgpu_init(const hfgpu_basis* B, hfgpu_handle** out) {
    if (!B || !out || B->nsh <= 0 || B->nb <= 0 || B->maxprim <= 0)
        return set_err(HFGPU_ERR_ARG, "hfgpu_init: bad arguments");
    *out = nullptr;
    hfgpu_handle* h = new hfgpu_handle();
    h->nsh = B->nsh;
    h->nb = B->nb;
    h->shtyp.assign(B->shtyp, B->shtyp + B->nsh);
    h->nzet.assign(B->nzet, B->nzet + B->nsh);
    h->aosh.assign(B->aosh, B->aosh + B->nsh);
    const int MP = B->maxprim;
    for (int s = 0; s < h->nsh; ++s) {
        int t = h->shtyp[s];
        if (t != HFGPU_SHELL_S && t != HFGPU_SHELL_P && t != HFGPU_SHELL_D && t != HFGPU_SHELL_L) {
            delete h;
            return set_err(HFGPU_ERR_ARG, "hfgpu_init: unknown shell type " + std::to_string(t));
        }
        if (h->nzet[s] < 1 || h->nzet[s] > MP) {
            delete h;
            return set_err(HFGPU_ERR_ARG, "hfgpu_init: bad primitive count");
        }
    }
    std::vector<GPrim> prims;
    std::vector<HostPair> plist[NPT];
    h->npairs = build_pairs(B, plist, prims, h->refcount);
    for (int t = 0; t < NPT; ++t) h->pairs[t] = std::move(plist[t]);
    std::vector<double> bt;
    std::vector<float> btf;
    build_boys_table(bt, btf);
    cudaError_t ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        std::string m = std::string("cudaStreamCreate: ") + cudaGetErrorString(ce);
        delete h;
        return set_err(HFGPU_ERR_CUDA, m);
    }
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev);
        h->device = dev;
        if (h->nsm <= 0) h->nsm = 148;
        // eight blocks per SM; HFGPU_MERGE_BLOCKS overrides (0: one launch per
        // role always).  Served-size jobs, 200 at once on 8 slots, one box:
        // 10.8 jobs/s without merging, 14.9 at 2 x SMs, 23.9 at 8 x SMs
        h->merge_blocks = 8LL * h->nsm;
        if (const char* e = getenv("HFGPU_MERGE_BLOCKS")) h->merge_blocks = atoll(e);
        if (const char* e = getenv("HFGPU_STREAMS")) h->nstreams = std::max(1, std::min(NSTREAM, atoi(e)));
        if (const char* e = getenv("HFGPU_SCATTER"))  // "single" / "grouped" override the per-class choice
            h->grouped_scatter = strcmp(e, "single") == 0 ? 0 : strcmp(e, "grouped") == 0 ? 2 : 1;
    }
    int rc = 0;
    const size_t nb2 = (size_t)h->nb * h->nb;
    rc |= dalloc(&h->d_shtyp, h->nsh, h->stream);
    rc |= dalloc(&h->d_aosh, h->nsh, h->stream);
    rc |= dalloc(&h->d_psoa, 8 * std::max<size_t>(prims.size(), 1), h->stream);
    rc |= dalloc(&h->d_boys, bt.size(), h->stream);
    rc |= dalloc(&h->d_boysf, btf.size(), h->stream);
    rc |= dalloc(&h->d_P, nb2, h->stream);
    rc |= dalloc(&h->d_F, nb2, h->stream);
    rc |= dalloc(&h->d_G, nb2, h->stream);
    rc |= dalloc(&h->d_md, (size_t)h->nsh * h->nsh, h->stream);
    rc |= dalloc(&h->d_cnt, 2 * NCLS, h->stream);
    rc |= dalloc(&h->d_stats, NCLS, h->stream);
    rc |= dalloc(&h->d_ncls, 2 * NCLS, h->stream);
    rc |= dalloc(&h->d_Pb, nb2, h->stream);
    rc |= dalloc(&h->d_boff, (size_t)h->nsh * h->nsh, h->stream);
    rc |= dalloc(&h->d_aomap, (size_t)h->nb, h->stream);
    rc |= dalloc(&h->d_nfsh, (size_t)h->nsh, h->stream);
    for (int t = 0; t < NPT; ++t) {
        size_t n = h->pairs[t].size();
        rc |= dalloc(&h->d_pairs[t], n, h->stream);
        rc |= dalloc(&h->d_schw[t], n, h->stream);
        rc |= dalloc(&h->d_apairs[t], n, h->stream);
        rc |= dalloc(&h->d_ash[t], n, h->stream);
        rc |= dalloc(&h->d_aschw[t], n, h->stream);
    }
    if (rc) {
        hfgpu_finalize(h);
        return HFGPU_ERR_NOMEM;
    }
    for (int i = 0; i < 2 * NCLS + 2; ++i) cudaEventCreate(&h->ev[i]);
    cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
    for (int k = 0; k < NSTREAM; ++k) {
        cudaStreamCreateWithFlags(&h->aux[k], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&h->join[k], cudaEventDisableTiming);
    }
    // uploads on the handle's own stream (pageable sources are staged before
    // the call returns); one synchronisation of that stream at the end
    auto up = [&](void* d, const void* s, size_t bytes) {
        if (bytes == 0) return cudaSuccess;
        return cudaMemcpyAsync(d, s, bytes, cudaMemcpyHostToDevice, h->stream);
    };
    ce = up(h->d_shtyp, h->shtyp.data(), h->nsh * sizeof(int));
    if (ce == cudaSuccess) ce = up(h->d_aosh, h->aosh.data(), h->nsh * sizeof(int));
    if (ce == cudaSuccess) {
        std::vector<double> soa = prims_soa(prims);
        ce = up(h->d_psoa, soa.data(), soa.size() * sizeof(double));
        h->psoa = soa_view(h->d_psoa, prims.size());
    }
    h->hprims = prims;
    if (ce == cudaSuccess) ce = up(h->d_boys, bt.data(), bt.size() * sizeof(double));
    if (ce == cudaSuccess) ce = up(h->d_boysf, btf.data(), btf.size() * sizeof(float));
    {  // shell-pair block layout of the density
        auto nf = [](int t) { return t == HFGPU_SHELL_S ? 1 : t == HFGPU_SHELL_P ? 3 : t == HFGPU_SHELL_D ? 5 : 4; };
        std::vector<int> nfsh(h->nsh), boff((size_t)h->nsh * h->nsh);
        std::vector<int2> aomap(h->nb, make_int2(0, 0));
        for (int a = 0; a < h->nsh; ++a) {
            nfsh[a] = nf(h->shtyp[a]);
            for (int i = 0; i < nfsh[a] && h->aosh[a] + i < h->nb; ++i) aomap[h->aosh[a] + i] = make_int2(a, i);
        }
        long long off = 0;
        for (int a = 0; a < h->nsh; ++a)
            for (int b = 0; b < h->nsh; ++b) {
                boff[(size_t)a * h->nsh + b] = (int)off;
                off += (long long)nfsh[a] * nfsh[b];
            }
        if (off != (long long)h->nb * h->nb) ce = cudaErrorInvalidValue;  // the shells must tile the basis
        if (ce == cudaSuccess) ce = up(h->d_nfsh, nfsh.data(), nfsh.size() * sizeof(int));
        if (ce == cudaSuccess) ce = up(h->d_boff, boff.data(), boff.size() * sizeof(int));
        if (ce == cudaSuccess) ce = up(h->d_aomap, aomap.data(), aomap.size() * sizeof(int2));
    }
    for (int t = 0; t < NPT && ce == cudaSuccess; ++t) {
        std::vector<GPair> gp(h->pairs[t].size());
        for (size_t i = 0; i < gp.size(); ++i) gp[i] = h->pairs[t][i].g;
        ce = up(h->d_pairs[t], gp.data(), gp.size() * sizeof(GPair));
    }
    if (ce != cudaSuccess) {
        std::string m = std::string("hfgpu_init upload: ") + cudaGetErrorString(ce);
        hfgpu_finalize(h);
        return set_err(HFGPU_ERR_CUDA, m);
    }
    // staged diagonal builders: (i, i) lists (their scratch is sized by the
    // handle's budget at the first fock_build_initial_diag)
    {
        for (int t = 0; t < NPT && ce == cudaSuccess; ++t) {
            const ClassKernels& K = CLASS_KERNELS[class_index(t, t)];
            const size_t n = h->pairs[t].size();
            if (K.mode == 0 || n == 0) continue;
            std::vector<uint2> dl(n);
            for (size_t i = 0; i < n; ++i) dl[i] = make_uint2((unsigned)i, (unsigned)i);
            if (dalloc(&h->d_diaglist[t], n, h->stream)) {
                hfgpu_finalize(h);
                return HFGPU_ERR_NOMEM;
            }
            ce = cudaMemcpyAsync(h->d_diaglist[t], dl.data(), n * sizeof(uint2), cudaMemcpyHostToDevice, h->stream);
        }
    }
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_stats, 0, NCLS * sizeof(ClassStats), h->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_ncls, 0, 2 * NCLS * sizeof(unsigned long long), h->stream);
    // the handle's own stream only: other handles' work on the device goes on
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) {
        std::string m = std::string("hfgpu_init: ") + cudaGetErrorString(ce);
        hfgpu_finalize(h);
        return set_err(HFGPU_ERR_CUDA, m);
    }
    *out = h;
    return HFGPU_OK;
}

int hfgpu_finalize(hfgpu_handle* h) {
    if (!h) return HFGPU_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    void* bufs[] = {h->d_shtyp, h->d_aosh, h->d_psoa, h->d_apsoa, h->d_boys, h->d_boysf, h->d_P, h->d_F, h->d_G,
                    h->d_md, h->d_subs, h->d_q, h->d_cnt, h->d_stats, h->d_scratch, h->d_dscratch,
                    h->d_ncls, h->d_Pb, h->d_boff, h->d_aomap, h->d_nfsh};
    for (void* b : bufs)
        if (b) cudaFreeAsync(b, h->stream);
    for (int t = 0; t < NPT; ++t) {
        void* tb[] = {h->d_pairs[t], h->d_schw[t], h->d_apairs[t], h->d_ash[t], h->d_aschw[t], h->d_diaglist[t]};
        for (void* b : tb)
            if (b) cudaFreeAsync(b, h->stream);
    }
    for (int i = 0; i < 2 * NCLS + 2; ++i)
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    for (int k = 0; k < NSTREAM; ++k) {
        if (h->aux[k]) {
            cudaStreamSynchronize(h->aux[k]);
            cudaStreamDestroy(h->aux[k]);
        }
        if (h->join[k]) cudaEventDestroy(h->join[k]);
    }
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);  // the stream-ordered frees above
        cudaStreamDestroy(h->stream);
    }
    delete h;
    return HFGPU_OK;
}

// Scratch of the staged diagonal builders (one chunk of stride pairs holds
// accumulators, outputs and role maxima per pair), sized once per handle by
// its scratch budget (hfgpu_set_scratch_budget, else the default).
static int alloc_diag_scratch(hfgpu_handle* h) {
    if (h->d_dscratch) return HFGPU_OK;
    const size_t budget = h->scratch_budget ? h->scratch_budget / sizeof(double) : scratch_budget_doubles();
    size_t need = 0;
    for (int t = 0; t < NPT; ++t) {
        const ClassKernels& K = CLASS_KERNELS[class_index(t, t)];
        const size_t n = h->pairs[t].size();
        if (K.mode == 0 || n == 0) continue;
        const size_t per = (size_t)K.nacc + K.nout + K.nrole_b;
        const size_t st = (std::max<size_t>(std::min<size_t>(n, budget / per), TQ) + TQ - 1) / TQ * TQ;  // whole tiles
        h->dstride[t] = st;
        need = std::max(need, st * per);
    }
    if (!need) return HFGPU_OK;
    const int rc = dalloc(&h->d_dscratch, need, h->stream);
    if (rc == HFGPU_OK) h->dscratch_doubles = need;
    return rc;
}

static void drop_graph(hfgpu_handle* h) {
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
}

int hfgpu_fock_build_initial_diag(hfgpu_handle* h, double* f, const double* p, double thr) {
    if (!h || !f || !p) return set_err(HFGPU_ERR_ARG, "null argument");
    {
        HF_DEVICE_LOCK;
        drop_graph(h);  // the Schwarz pass re-sizes the buffers a captured build points at
        const int rc = alloc_diag_scratch(h);
        if (rc) return rc;
    }
    int rc = upload_fp(h, f, p);
    if (rc) return rc;
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    rc = launch_diag(h, 0, h->d_P, thr);
    if (rc) return rc;
    rc = launch_symm(h, h->d_F);
    if (rc) return rc;
    rc = download_f(h, f);
    if (rc) return rc;
    return build_active(h);
}

int hfgpu_fock_build_diag(hfgpu_handle* h, double* f, const double* p, double thr) {
    if (!h || !f || !p) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    int rc = upload_fp(h, f, p);
    if (rc) return rc;
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    if ((rc = launch_maxdm(h, h->d_P))) return rc;
    if ((rc = launch_diag(h, 1, h->d_P, thr))) return rc;
    if ((rc = launch_symm(h, h->d_F))) return rc;
    return download_f(h, f);
}

static int non_diag_host(hfgpu_handle* h, double* f, const double* p, double thr, int jonly, double f32cut) {
    if (!h || !f || !p) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    int rc = upload_fp(h, f, p);
    if (rc) return rc;
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    if ((rc = launch_maxdm(h, h->d_P))) return rc;
    if ((rc = run_non_diag(h, h->d_P, thr, jonly, f32cut))) return rc;
    if ((rc = launch_symm(h, h->d_F))) return rc;
    return download_f(h, f);
}

int hfgpu_fock_build_non_diag(hfgpu_handle* h, double* f, const double* p, double thr) {
    return non_diag_host(h, f, p, thr, 0, 0.0);
}

int hfgpu_fock_build_non_diag_j_only(hfgpu_handle* h, double* f, const double* p, double thr) {
    return non_diag_host(h, f, p, thr, 1, 0.0);
}

int hfgpu_fock_build_non_diag_mixed(hfgpu_handle* h, double* f, const double* p, double thr, double fp32_cutoff) {
    return non_diag_host(h, f, p, thr, 0, fp32_cutoff);
}

static int device_build(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag, double thr_non_diag,
                        double fp32_cutoff, bool capture) {
    int rc;
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    if ((rc = launch_maxdm(h, p_dev))) return rc;
    if ((rc = launch_diag(h, 1, p_dev, thr_diag))) return rc;
    if ((rc = run_non_diag(h, p_dev, thr_non_diag, 0, fp32_cutoff, capture))) return rc;
    return launch_symm(h, f_dev);
}

int hfgpu_fock_build_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag,
                            double thr_non_diag, double fp32_cutoff) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    return device_build(h, f_dev, p_dev, thr_diag, thr_non_diag, fp32_cutoff, false);
}

int hfgpu_fock_build_initial_diag_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    {
        HF_DEVICE_LOCK;
        drop_graph(h);  // the Schwarz pass re-sizes the buffers a captured build points at
        const int rc = alloc_diag_scratch(h);
        if (rc) return rc;
    }
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    int rc = launch_diag(h, 0, p_dev, thr);
    if (rc) return rc;
    if ((rc = launch_symm(h, f_dev))) return rc;
    return build_active(h);  // reads the Schwarz factors back (synchronises the handle's stream)
}

int hfgpu_fock_build_non_diag_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr,
                                     double fp32_cutoff) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    HF_CHECK(cudaMemsetAsync(h->d_G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    int rc;
    if ((rc = launch_maxdm(h, p_dev))) return rc;
    if ((rc = run_non_diag(h, p_dev, thr, 0, fp32_cutoff))) return rc;
    return launch_symm(h, f_dev);
}

int hfgpu_graph_capture(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag, double thr_non_diag,
                        double fp32_cutoff) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    HF_CHECK(cudaStreamSynchronize(h->stream));
    HF_DEVICE_LOCK;  // held from the start of the capture to its end
    drop_graph(h);
    const long long before = h->launches;
    // thread-local mode: other host threads (other jobs, the caller's own
    // framework) may keep allocating while this thread records
    HF_CHECK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = device_build(h, f_dev, p_dev, thr_diag, thr_non_diag, fp32_cutoff, true);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->stream, &g);  // always ends the capture
    if (rc != HFGPU_OK || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (rc != HFGPU_OK) return rc;
        return set_err(HFGPU_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
    }
    h->graph = g;
    h->graph_launches = h->launches - before;
    h->launches = before;  // recorded, not run
    h->gkey_f = f_dev;
    h->gkey_p = p_dev;
    h->gkey_thr[0] = thr_diag;
    h->gkey_thr[1] = thr_non_diag;
    h->gkey_thr[2] = fp32_cutoff;
    const cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
    if (ie != cudaSuccess) {
        h->gexec = nullptr;
        drop_graph(h);
        return set_err(HFGPU_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
    }
    return HFGPU_OK;
}

int hfgpu_graph_launch(hfgpu_handle* h) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    if (!h->gexec) return set_err(HFGPU_ERR_STATE, "hfgpu_graph_capture has not been called");
    HF_CHECK(cudaGraphLaunch(h->gexec, h->stream));
    h->launches += h->graph_launches;
    return HFGPU_OK;
}

// Enqueue one device build on the caller's stream with no host round trip
// (launches sized as for a capture), so that a caller's own CUDA-graph
// capture of a whole SCF iteration can include it.
int hfgpu_fock_build_device_on(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag,
                               double thr_non_diag, double fp32_cutoff, void* stream) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    cudaStream_t own = h->stream;
    h->stream = (cudaStream_t)stream;  // the build forks from and joins back to this stream
    const int rc = device_build(h, f_dev, p_dev, thr_diag, thr_non_diag, fp32_cutoff, true);
    h->stream = own;
    return rc;
}

// Solves the (n x n) system A x = b in place of b on the device (Gaussian
// elimination with partial pivoting, one thread): the DIIS equations of a
// device-resident SCF step, n <= 32.  A is row-major and is overwritten.
__global__ void k_small_solve(double* A, double* b, int n, int* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int ok = 1;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (fabs(A[r * n + c]) > fabs(A[piv * n + c])) piv = r;
        if (A[piv * n + c] == 0.0) { ok = 0; break; }
        if (piv != c) {
            for (int k = 0; k < n; ++k) { const double t = A[c * n + k]; A[c * n + k] = A[piv * n + k]; A[piv * n + k] = t; }
            const double t = b[c]; b[c] = b[piv]; b[piv] = t;
        }
        for (int r = c + 1; r < n; ++r) {
            const double m = A[r * n + c] / A[c * n + c];
            for (int k = c; k < n; ++k) A[r * n + k] -= m * A[c * n + k];
            b[r] -= m * b[c];
        }
    }
    if (ok)
        for (int r = n - 1; r >= 0; --r) {
            double s = b[r];
            for (int k = r + 1; k < n; ++k) s -= A[r * n + k] * b[k];
            b[r] = s / A[r * n + r];
        }
    if (status) *status = ok;
}

int hfgpu_small_solve(double* a_dev, double* b_dev, int n, int* status_dev, void* stream) {
    if (!a_dev || !b_dev || n <= 0 || n > 32) return set_err(HFGPU_ERR_ARG, "hfgpu_small_solve: bad arguments");
    k_small_solve<<<1, 32, 0, (cudaStream_t)stream>>>(a_dev, b_dev, n, status_dev);
    HF_CHECK(cudaGetLastError());
    return HFGPU_OK;
}

int hfgpu_fock_build_graph(hfgpu_handle* h, double* f, const double* p, double thr_diag, double thr_non_diag,
                           double fp32_cutoff) {
    if (!h || !f || !p) return set_err(HFGPU_ERR_ARG, "null argument");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    const bool same = h->gexec && h->gkey_f == h->d_F && h->gkey_p == h->d_P && h->gkey_thr[0] == thr_diag &&
                      h->gkey_thr[1] == thr_non_diag && h->gkey_thr[2] == fp32_cutoff;
    int rc;
    if (!same && (rc = hfgpu_graph_capture(h, h->d_F, h->d_P, thr_diag, thr_non_diag, fp32_cutoff))) return rc;
    if ((rc = upload_fp(h, f, p))) return rc;
    HF_CHECK(cudaGraphLaunch(h->gexec, h->stream));
    h->launches += h->graph_launches;
    return download_f(h, f);
}

int hfgpu_synchronize(hfgpu_handle* h) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    HF_CHECK(cudaStreamSynchronize(h->stream));
    return HFGPU_OK;
}

int hfgpu_batch_create(hfgpu_handle* const* hs, int n, hfgpu_batch** out) {
    if (!hs || !out || n <= 0) return set_err(HFGPU_ERR_ARG, "hfgpu_batch_create: bad arguments");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!hs[i]) return set_err(HFGPU_ERR_ARG, "hfgpu_batch_create: null handle");
        if (!hs[i]->graph)
            return set_err(HFGPU_ERR_STATE, "hfgpu_batch_create: handle " + std::to_string(i) +
                                                " has no captured build (call hfgpu_graph_capture)");
        for (int j = 0; j < i; ++j)
            if (hs[j] == hs[i]) return set_err(HFGPU_ERR_ARG, "hfgpu_batch_create: a handle appears twice");
    }
    HF_DEVICE_LOCK;
    hfgpu_batch* b = new hfgpu_batch();
    b->hs.assign(hs, hs + n);
    cudaError_t ce = cudaGraphCreate(&b->graph, 0);
    // one child graph per instance, no edges between them: the instances
    // share nothing on the device and run concurrently
    for (int i = 0; i < n && ce == cudaSuccess; ++i) {
        cudaGraphNode_t node;
        ce = cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, hs[i]->graph);
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (ce != cudaSuccess) {
        hfgpu_batch_destroy(b);
        return set_err(HFGPU_ERR_CUDA, std::string("hfgpu_batch_create: ") + cudaGetErrorString(ce));
    }
    *out = b;
    return HFGPU_OK;
}

int hfgpu_batch_launch(hfgpu_batch* b, void* stream) {
    if (!b || !b->exec) return set_err(HFGPU_ERR_ARG, "null batch");
    HF_CHECK(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    for (hfgpu_handle* h : b->hs) h->launches += h->graph_launches;
    return HFGPU_OK;
}

int hfgpu_batch_destroy(hfgpu_batch* b) {
    if (!b) return HFGPU_OK;
    HF_DEVICE_LOCK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    delete b;
    return HFGPU_OK;
}

int hfgpu_set_scratch_budget(hfgpu_handle* h, size_t bytes) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    if (h->have_schwarz) return set_err(HFGPU_ERR_STATE, "set the scratch budget before fock_build_initial_diag");
    h->scratch_budget = bytes;
    return HFGPU_OK;
}

int hfgpu_device_bytes(const hfgpu_handle* h, size_t* bytes) {
    if (!h || !bytes) return set_err(HFGPU_ERR_ARG, "null argument");
    size_t b = 0;
    const size_t nb2 = (size_t)h->nb * h->nb;
    b += 4 * nb2 * sizeof(double);                            // P, F, G, blocked P
    b += ((size_t)h->nsh * h->nsh + 2 * (size_t)h->nb + h->nsh) * sizeof(int);
    b += (size_t)h->nsh * h->nsh * sizeof(double);            // maxdm
    b += 2 * (size_t)h->nsh * sizeof(int);
    b += 8 * h->hprims.size() * sizeof(double);               // all-pairs primitives
    for (int t = 0; t < NPT; ++t) {
        const size_t n = h->pairs[t].size();
        b += n * (2 * sizeof(GPair) + sizeof(double) * 2 + sizeof(int2) + (h->d_diaglist[t] ? sizeof(uint2) : 0));
    }
    b += 8 * h->naprims * sizeof(double);                     // active-list primitives
    b += h->qcap * sizeof(uint2);                             // quartet lists
    b += h->scratch_doubles * sizeof(double);                 // staged scratch
    b += h->dscratch_doubles * sizeof(double);                // staged diagonal builders' scratch
    b += h->subcap * (sizeof(ScreenSub) + 2 * sizeof(unsigned long long));
    b += (size_t)(BOYS_MMAX + 1) * BOYS_BLK * (sizeof(double) + sizeof(float));
    *bytes = b;
    return HFGPU_OK;
}

int hfgpu_dims(const hfgpu_handle* h, int* nb, int* nsh, int* npairs) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    if (nb) *nb = h->nb;
    if (nsh) *nsh = h->nsh;
    if (npairs) *npairs = h->npairs;
    return HFGPU_OK;
}

int hfgpu_get_schwarz(const hfgpu_handle* h, double* schw_sh, int* last) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    if (schw_sh) {
        for (int t = 0; t < NPT; ++t)
            for (size_t i = 0; i < h->pairs[t].size(); ++i) {
                const GPair& g = h->pairs[t][i].g;
                schw_sh[(size_t)g.sa * h->nsh + g.sb] = h->schw[t][i];
                schw_sh[(size_t)g.sb * h->nsh + g.sa] = h->schw[t][i];
            }
    }
    if (last)
        for (int c = 0; c < 10; ++c) last[c] = h->last_ref[c];
    return HFGPU_OK;
}

int hfgpu_get_class_stats(const hfgpu_handle* h, long long* n_pass, long long* n_scattered, long long* n_prim,
                          long long* n_fp32, double* ms) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    // the counters live on the device (a captured build never returns to the
    // host); read them after the handle's stream has drained
    ClassStats st[NCLS];
    unsigned long long cnt[2 * NCLS];
    HF_DEVICE_LOCK;
    HF_CHECK(cudaStreamSynchronize(h->stream));
    HF_CHECK(cudaMemcpy(st, h->d_stats, sizeof(st), cudaMemcpyDeviceToHost));
    HF_CHECK(cudaMemcpy(cnt, h->d_ncls, sizeof(cnt), cudaMemcpyDeviceToHost));
    for (int c = 0; c < NCLS; ++c) {
        if (n_pass) n_pass[c] = (long long)(cnt[2 * c] + cnt[2 * c + 1]);
        if (n_scattered) n_scattered[c] = (long long)st[c].scattered;
        if (n_prim) n_prim[c] = (long long)st[c].prim;
        if (n_fp32) n_fp32[c] = (long long)st[c].fp32;
        if (ms) ms[c] = h->st_ms[c];
    }
    return HFGPU_OK;
}

int hfgpu_launch_count(const hfgpu_handle* h, long long* n) {
    if (!h || !n) return set_err(HFGPU_ERR_ARG, "null argument");
    *n = h->launches;
    return HFGPU_OK;
}

int hfgpu_set_timing(hfgpu_handle* h, int on) {
    if (!h) return set_err(HFGPU_ERR_ARG, "null handle");
    h->timing = on;
    return HFGPU_OK;
}

void* hfgpu_stream(hfgpu_handle* h) { return h ? (void*)h->stream : nullptr; }

int hfgpu_measure_fma_peak(double* fp64_gflops, double* fp32_gflops) {
    HF_DEVICE_LOCK;
    int dev = 0, nsm = 0;
    HF_CHECK(cudaGetDevice(&dev));
    HF_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double* dd = nullptr;
    HF_CHECK(cudaMalloc(&dd, 64));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
    double res[2] = {0, 0};
    for (int prec = 0; prec < 2; ++prec) {
        float best = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(e0);
            if (prec == 0) k_fma_peak<double><<<blocks, threads>>>(dd, iters, 0.999999, 1e-7);
            else k_fma_peak<float><<<blocks, threads>>>((float*)dd, iters, 0.999999f, 1e-7f);
            cudaEventRecord(e1);
            cudaError_t ce = cudaEventSynchronize(e1);
            if (ce != cudaSuccess) {
                cudaFree(dd);
                g_err = cudaGetErrorString(ce);
                return HFGPU_ERR_CUDA;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) best = std::min(best, ms);
        }
        res[prec] = 2.0 * 8.0 * (double)iters * threads * blocks / (best * 1e-3) / 1e9;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dd);
    if (fp64_gflops) *fp64_gflops = res[0];
    if (fp32_gflops) *fp32_gflops = res[1];
    return HFGPU_OK;
}

}  // extern "C"

// ------------------------------------------------ no-allocation variant ----
// Scratch of hfgpu_fock_build_diag_static: the one-triangle accumulation
// buffer G (nb x nb) and the shell-pair density maxima (nsh x nsh) live in
// this file-scope device array instead of memory from cudaMalloc.  Every GPU
// that loads the library holds it (10,485,760 bytes, 10.0 MiB) until the process exits.
namespace {
constexpr int STATIC_MAX_NB = 1024;
constexpr int STATIC_MAX_NSH = 512;
constexpr size_t STATIC_SCRATCH_DOUBLES =
    (size_t)STATIC_MAX_NB * STATIC_MAX_NB + (size_t)STATIC_MAX_NSH * STATIC_MAX_NSH;
}  // namespace

static __device__ __align__(256) double g_static_scratch[STATIC_SCRATCH_DOUBLES];

namespace {
constexpr int STATIC_MAX_DEVICES = 64;
std::mutex g_static_mu;
double* g_static_ptr[STATIC_MAX_DEVICES] = {};

// Device address of g_static_scratch on the current device.  Host code sees
// only a host-side stand-in under that name, so the address is looked up once
// per device, with that device current, and cached.
int static_scratch(double** out) {
    int dev = 0;
    HF_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= STATIC_MAX_DEVICES) return set_err(HFGPU_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return set_err(HFGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(g_static_scratch): ") +
                                               cudaGetErrorString(e));
        g_static_ptr[dev] = (double*)p;
    }
    *out = g_static_ptr[dev];
    return HFGPU_OK;
}
}  // namespace

extern "C" int hfgpu_fock_build_diag_static(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr) {
    if (!h || !f_dev || !p_dev) return set_err(HFGPU_ERR_ARG, "null argument");
    if (h->nb > STATIC_MAX_NB || h->nsh > STATIC_MAX_NSH)
        return set_err(HFGPU_ERR_ARG, "hfgpu_fock_build_diag_static: nb " + std::to_string(h->nb) + " / nsh " +
                                          std::to_string(h->nsh) + " exceeds the static scratch limit of nb <= " +
                                          std::to_string(STATIC_MAX_NB) + ", nsh <= " +
                                          std::to_string(STATIC_MAX_NSH));
    if (!h->have_schwarz) return set_err(HFGPU_ERR_STATE, "fock_build_initial_diag has not been called");
    {
        int dev = -1;
        HF_CHECK(cudaGetDevice(&dev));
        if (dev != h->device)
            return set_err(HFGPU_ERR_ARG, "hfgpu_fock_build_diag_static: the current device (" + std::to_string(dev) +
                                              ") is not the device the handle was created on (" +
                                              std::to_string(h->device) + ")");
    }
    double* scratch = nullptr;
    int rc = static_scratch(&scratch);
    if (rc) return rc;
    double* G = scratch;
    double* md = scratch + (size_t)STATIC_MAX_NB * STATIC_MAX_NB;
    // G keeps the previous call's sums: clear it first
    HF_CHECK(cudaMemsetAsync(G, 0, (size_t)h->nb * h->nb * sizeof(double), h->stream));
    if ((rc = launch_maxdm(h, p_dev, md))) return rc;
    if ((rc = launch_diag(h, 1, p_dev, thr, G, md))) return rc;
    return launch_symm(h, f_dev, G);
}
