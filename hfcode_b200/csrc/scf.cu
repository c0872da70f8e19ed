// Device-resident RHF step: the reference's SCF protocol
// (direct_hartreefock.f90:1-234) with every matrix of a job in the GPU's
// memory and the cycle driven from C++ on the builder handle's stream.
//
//   Fock builds        this library (device-pointer entry points of hfgpu.h)
//   E_elec, DIIS rows  one pass over the matrices (k_cycle_scalars) into device scalars
//   F P S - S P F, X^T R X, X F X^T, C = X C', P = 2 C_occ C_occ^T   cuBLAS dgemm/geam
//   the density        SP2 purification (cuBLAS dgemm); cuSOLVER syevd where
//                      eigenvectors are needed (core guess, level shift, orbital energies)
//   max |R|, max |dP|  the same pass
//
// The host reads one small block of scalars per cycle (two dots, the new
// DIIS row, two maxima) and takes the protocol's decisions as the reference
// does; the bordered DIIS system (at most 9 x 9) is solved on the host.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hfgpu_scf.h"

namespace hfgpu {
void set_last_error(const std::string& msg);
std::recursive_mutex& device_mutex();
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);  // the library's memory pool
}  // namespace hfgpu

namespace {

constexpr int NDIIS = 8;              // direct_hartreefock.f90:13
constexpr double INTTHRESH = 1e-10;   // molprops.f90:162

// Scalars of one cycle, read back together.
struct CycleScalars {
    double ph, pf;                 // sum P H, sum P F
    double brow[NDIIS];            // <R_new, R_j> over the history slots
    unsigned long long resmax;     // max |R| as the bits of a non-negative double
    unsigned long long dpmax;      // max |P - Pold|
};

// out[:, j] = v[:, j] / sqrt(w[j]) (columns of an n x n column-major matrix)
__global__ void k_scale_cols(const double* __restrict__ v, const double* __restrict__ w, double* __restrict__ out,
                             int n) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)n * n) return;
    out[t] = v[t] / sqrt(w[t / n]);
}

// Gershgorin discs of a symmetric n x n matrix, one warp per row (read as
// the column, which is contiguous): lo[i] = a_ii - r_i, hi[i] = a_ii + r_i,
// r_i = sum_{j != i} |a_ij|
__global__ void k_gershgorin_rows(const double* __restrict__ a, int n, double* __restrict__ lo,
                                  double* __restrict__ hi) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n) return;
    const double* col = a + (size_t)i * n;
    double r = 0.0;
    for (int j = lane; j < n; j += 32)
        if (j != i) r += fabs(col[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (lane == 0) {
        lo[i] = col[i] - r;
        hi[i] = col[i] + r;
    }
}

// bounds[0] = min lo, bounds[1] = max hi (one block of 1024 threads)
__global__ void k_gershgorin_bounds(const double* __restrict__ lo, const double* __restrict__ hi, int n,
                                    double* bounds) {
    __shared__ double slo[1024], shi[1024];
    double a = 1e300, b = -1e300;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a = fmin(a, lo[i]);
        b = fmax(b, hi[i]);
    }
    slo[threadIdx.x] = a;
    shi[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            slo[threadIdx.x] = fmin(slo[threadIdx.x], slo[threadIdx.x + o]);
            shi[threadIdx.x] = fmax(shi[threadIdx.x], shi[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bounds[0] = slo[0];
        bounds[1] = shi[0];
    }
}

// Block sums of two values into acc[0], acc[1] with one atomic each.
__device__ __forceinline__ void block_add2(double a, double b, double* acc) {
    __shared__ double sa[32], sb[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            atomicAdd(acc, a);
            atomicAdd(acc + 1, b);
        }
    }
}

// X = (hi I - F) / (hi - lo): the start of the purification, spectrum in [0, 1]
// with the occupied orbitals (lowest energies) nearest 1.  Adds tr X and
// ||X||_F^2 (= tr X^2, X symmetric) into tr[0], tr[1] (zeroed before).
__global__ void k_sp2_start(const double* __restrict__ f, const double* __restrict__ bounds, double* __restrict__ x,
                            int n, double* tr) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    double d = 0.0, q = 0.0;
    if (t < (size_t)n * n) {
        const double lo = bounds[0], hi = bounds[1];
        const int i = (int)(t % n), j = (int)(t / n);
        const double v = ((i == j ? hi : 0.0) - f[t]) / (hi - lo);
        x[t] = v;
        d = i == j ? v : 0.0;
        q = v * v;
    }
    block_add2(d, q, tr);
}

// One SP2 step: X <- X^2 when that brings the trace nearer nocc, else
// X <- 2X - X^2 (tr(2X - X^2) = 2 tr X - tr X^2), decided from tr_in (tr X,
// tr X^2 of the current X).  Adds the new X's traces into tr_out and clears
// tr_clear, the slot the next step adds into.
__global__ void k_sp2_update(double* __restrict__ x, const double* __restrict__ x2, const double* __restrict__ tr_in,
                             double* tr_out, double* tr_clear, double nocc, int n) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t == 0) {
        tr_clear[0] = 0.0;
        tr_clear[1] = 0.0;
    }
    double d = 0.0, q = 0.0;
    if (t < (size_t)n * n) {
        const bool square = fabs(tr_in[1] - nocc) < fabs(2.0 * tr_in[0] - tr_in[1] - nocc);
        const double v = square ? x2[t] : 2.0 * x[t] - x2[t];
        x[t] = v;
        d = (t % n) == (t / n) ? v : 0.0;
        q = v * v;
    }
    block_add2(d, q, tr_out);
}

// The cycle's scalars in one pass: sum P H, sum P F, <R_new, R_j> for the
// eight history slots, max |R_new| and max |P - Pold|, into out (zeroed).
struct CycleArgs {
    const double* P;
    const double* H;
    const double* F;
    const double* R;
    const double* Rj[8];
    const double* Pold;
    size_t n;
};
__global__ void k_cycle_scalars(CycleArgs c, CycleScalars* out) {
    double ph = 0.0, pf = 0.0, br[8] = {}, rm = 0.0, dm = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < c.n; i += (size_t)gridDim.x * blockDim.x) {
        const double p = c.P[i], r = c.R[i];
        ph += p * c.H[i];
        pf += p * c.F[i];
#pragma unroll
        for (int k = 0; k < 8; ++k) br[k] += r * c.Rj[k][i];
        rm = fmax(rm, fabs(r));
        dm = fmax(dm, fabs(p - c.Pold[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ph += __shfl_xor_sync(0xffffffffu, ph, o);
        pf += __shfl_xor_sync(0xffffffffu, pf, o);
#pragma unroll
        for (int k = 0; k < 8; ++k) br[k] += __shfl_xor_sync(0xffffffffu, br[k], o);
        rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, o));
        dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out->ph, ph);
        atomicAdd(&out->pf, pf);
#pragma unroll
        for (int k = 0; k < 8; ++k) atomicAdd(&out->brow[k], br[k]);
        atomicMax(&out->resmax, (unsigned long long)__double_as_longlong(rm));
        atomicMax(&out->dpmax, (unsigned long long)__double_as_longlong(dm));
    }
}

int fail(int code, const std::string& msg) {
    hfgpu::set_last_error(msg);
    return code;
}

}  // namespace

struct hfgpu_scf {
    hfgpu_handle* h = nullptr;
    int nb = 0, nocc = 0;
    double enuc = 0.0;
    cudaStream_t st = nullptr;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t sol = nullptr;
    // device matrices (nb x nb)
    double *S = nullptr, *H = nullptr, *X = nullptr, *P = nullptr, *Pold = nullptr, *F = nullptr, *Fprev = nullptr;
    double *dP = nullptr, *dF = nullptr, *T1 = nullptr, *T2 = nullptr, *Fob = nullptr, *Cob = nullptr;
    double* R[NDIIS] = {};      // residual history (slots)
    double* FO[NDIIS] = {};     // orthogonalised Fock history (slots)
    double* W = nullptr;        // eigenvalues
    double* work = nullptr;     // syevd workspace
    int lwork = 0;
    int* info = nullptr;
    void* blas_ws = nullptr;
    void* arena = nullptr;       // one stream-ordered allocation holding every buffer above
    CycleScalars* sc = nullptr;  // device
    double* aux = nullptr;       // purification: bounds[2], trace slots[6], then row bounds lo[nb], hi[nb]
    bool eigs_current = false;   // W/eigs describe the last Fob
    size_t bytes = 0;
    // protocol state, carried from one hfgpu_scf_run call to the next
    double eelec = 0.0;
    bool have_cob = false;       // Cob holds the eigenvectors of the last eigensolve
    bool uselevshft = false;
    std::vector<double> eigs;    // host copy of the last eigenvalues
    int it = 0;                  // cycles done
    bool diis = false, fullfock = true, converged = false;
    int nusediis = 0, nfull = 0, nfullb = 0, ndelta = 0;
    double thresh = 0.0, deltae = 0.0, deltap = 0.0;
    int sp2_steps = 0;
    double ms_build = 0.0, ms_density = 0.0;
    cudaEvent_t ev[4] = {};      // build start/end, density start/end of the current cycle
    int slot[NDIIS] = {};        // history position -> buffer (position 0: newest)
    double eo[NDIIS] = {};       // energies of the history positions
    double B[NDIIS][NDIIS] = {}; // <R_j, R_k> by history position
};

namespace {

#define SCF_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(HFGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define SCF_BLAS(call)                                                                         \
    do {                                                                                       \
        cublasStatus_t s_ = (call);                                                            \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                       \
            return fail(HFGPU_ERR_CUDA, std::string(#call) + ": cuBLAS status " + std::to_string((int)s_)); \
    } while (0)
#define SCF_SOLVER(call)                                                                       \
    do {                                                                                       \
        cusolverStatus_t s_ = (call);                                                          \
        if (s_ != CUSOLVER_STATUS_SUCCESS)                                                     \
            return fail(HFGPU_ERR_CUDA, std::string(#call) + ": cuSOLVER status " + std::to_string((int)s_)); \
    } while (0)
#define SCF_RC(call)            \
    do {                        \
        int r_ = (call);        \
        if (r_) return r_;      \
    } while (0)

// C = alpha op(A) op(B) + beta C, all nb x nb
int gemm(hfgpu_scf* s, bool ta, bool tb, double alpha, const double* A, const double* B, double beta, double* C) {
    const int n = s->nb;
    SCF_BLAS(cublasDgemm(s->blas, ta ? CUBLAS_OP_T : CUBLAS_OP_N, tb ? CUBLAS_OP_T : CUBLAS_OP_N, n, n, n, &alpha, A,
                         n, B, n, &beta, C, n));
    return HFGPU_OK;
}

int copy(hfgpu_scf* s, double* dst, const double* src) {
    SCF_CUDA(cudaMemcpyAsync(dst, src, (size_t)s->nb * s->nb * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    return HFGPU_OK;
}

// Eigenvalues (W, ascending) and eigenvectors (Cob, columns) of the
// symmetric matrix A: the wrapper_dsyev role (wrapper_dsygv.f90:29-52).
int eigensolve(hfgpu_scf* s, const double* A) {
    SCF_RC(copy(s, s->Cob, A));
    SCF_SOLVER(cusolverDnDsyevd(s->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, s->nb, s->Cob, s->nb, s->W,
                                s->work, s->lwork, s->info));
    int info = 0;
    SCF_CUDA(cudaMemcpyAsync(&info, s->info, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    s->eigs.resize(s->nb);
    SCF_CUDA(cudaMemcpyAsync(s->eigs.data(), s->W, s->nb * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    SCF_CUDA(cudaStreamSynchronize(s->st));
    if (info != 0) return fail(HFGPU_ERR_CUDA, "syevd failed, info " + std::to_string(info));
    s->have_cob = true;
    return HFGPU_OK;
}

// P = 2 C_occ C_occ^T with C = X Cob (direct_hartreefock.f90:205,218)
int density_from_cob(hfgpu_scf* s, double* P) {
    SCF_RC(gemm(s, false, false, 1.0, s->X, s->Cob, 0.0, s->T1));
    const double two = 2.0, zero = 0.0;
    SCF_BLAS(cublasDgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_T, s->nb, s->nb, s->nocc, &two, s->T1, s->nb, s->T1, s->nb,
                         &zero, P, s->nb));
    return HFGPU_OK;
}

// P = 2 X D X^T from the orthogonalised Fock matrix Fo by second-order
// spectral projection (A. M. N. Niklasson, Phys. Rev. B 66, 155115 (2002)):
// D is the projector on the nocc lowest eigenvectors of Fo, the density the
// eigenvectors give (direct_hartreefock.f90:204-218), reached with matrix
// products only.  Each step's choice is made on the device; the host checks
// idempotency every few steps.
int density_by_purification(hfgpu_scf* s, const double* Fo, double* P) {
    const int nb = s->nb;
    const size_t n2 = (size_t)nb * nb;
    const unsigned blocks = (unsigned)((n2 + 255) / 256);
    double* X = s->T1;
    double* X2 = s->T2;
    double* bounds = s->aux;
    double* tr = s->aux + 2;  // three slots of (tr X, tr X^2), rotating with the steps
    double* lo = s->aux + 8;
    k_gershgorin_rows<<<(unsigned)((nb + 7) / 8), 256, 0, s->st>>>(Fo, nb, lo, lo + nb);
    k_gershgorin_bounds<<<1, 1024, 0, s->st>>>(lo, lo + nb, nb, bounds);
    SCF_CUDA(cudaMemsetAsync(tr, 0, 6 * sizeof(double), s->st));
    k_sp2_start<<<blocks, 256, 0, s->st>>>(Fo, bounds, X, nb, tr);
    SCF_CUDA(cudaGetLastError());
    // the first check after 16 steps (the start needs ~log2 of the spectral
    // range over the gap of them), then every 4; each step is the product X^2
    // and one update kernel that also forms the next step's traces
    constexpr int FIRST = 16, BLOCK = 4, MAXSTEP = 160;
    for (int step = 0; step < MAXSTEP;) {
        const int nstep = step == 0 ? FIRST : BLOCK;
        for (int k = 0; k < nstep; ++k) {
            const int q = step + k;
            SCF_RC(gemm(s, false, false, 1.0, X, X, 0.0, X2));
            k_sp2_update<<<blocks, 256, 0, s->st>>>(X, X2, tr + 2 * (q % 3), tr + 2 * ((q + 1) % 3),
                                                    tr + 2 * ((q + 2) % 3), (double)s->nocc, nb);
        }
        step += nstep;
        s->sp2_steps += nstep;
        SCF_CUDA(cudaGetLastError());
        double h_tr[2];
        SCF_CUDA(cudaMemcpyAsync(h_tr, tr + 2 * (step % 3), sizeof(h_tr), cudaMemcpyDeviceToHost, s->st));
        SCF_CUDA(cudaStreamSynchronize(s->st));
        // tr X - tr X^2 = sum x_k (1 - x_k) over the eigenvalues: zero for a projector
        if (std::fabs(h_tr[0] - h_tr[1]) < 1e-11 * std::max(1, s->nocc)) break;
    }
    // P = 2 X_s D X_s^T with X_s = S^-1/2
    SCF_RC(gemm(s, false, false, 1.0, s->X, X, 0.0, X2));
    SCF_RC(gemm(s, false, true, 2.0, X2, s->X, 0.0, P));
    return HFGPU_OK;
}

// Solves the bordered DIIS system A x = b in place (Gaussian elimination
// with partial pivoting; dsysv's role, wrapper_dsygv.f90:55-78).
bool small_solve(std::vector<double>& A, std::vector<double>& b, int n) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        if (A[piv * n + c] == 0.0) return false;
        if (piv != c) {
            for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[piv * n + k]);
            std::swap(b[c], b[piv]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double m = A[r * n + c] / A[c * n + c];
            for (int k = c; k < n; ++k) A[r * n + k] -= m * A[c * n + k];
            b[r] -= m * b[c];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double v = b[r];
        for (int k = r + 1; k < n; ++k) v -= A[r * n + k] * b[k];
        b[r] = v / A[r * n + r];
    }
    return true;
}

// cuBLAS / cuSOLVER handles are pooled across jobs: creating them costs
// milliseconds and may allocate, so a served job borrows a pair and gives it
// back when it ends.
struct LinAlg {
    cublasHandle_t blas;
    cusolverDnHandle_t sol;
};
std::mutex g_pool_mu;
std::vector<LinAlg> g_pool;

int acquire_linalg(hfgpu_scf* s) {
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (!g_pool.empty()) {
            s->blas = g_pool.back().blas;
            s->sol = g_pool.back().sol;
            g_pool.pop_back();
        }
    }
    if (!s->blas) {
        std::lock_guard<std::recursive_mutex> lk(hfgpu::device_mutex());  // creation may allocate
        SCF_BLAS(cublasCreate(&s->blas));
        SCF_SOLVER(cusolverDnCreate(&s->sol));
    }
    SCF_BLAS(cublasSetStream(s->blas, s->st));
    SCF_BLAS(cublasSetPointerMode(s->blas, CUBLAS_POINTER_MODE_HOST));
    SCF_SOLVER(cusolverDnSetStream(s->sol, s->st));
    return HFGPU_OK;
}

void release(hfgpu_scf* s) {
    if (s->st) cudaStreamSynchronize(s->st);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->arena) cudaFreeAsync(s->arena, s->st);
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->blas && s->sol) {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        g_pool.push_back({s->blas, s->sol});
    } else {
        if (s->blas) cublasDestroy(s->blas);
        if (s->sol) cusolverDnDestroy(s->sol);
    }
    delete s;
}

int create(hfgpu_handle* h, int nocc, double enuc, const double* S, const double* hcore, const double* p_guess,
           hfgpu_scf* s) {
    int nb = 0;
    SCF_RC(hfgpu_dims(h, &nb, nullptr, nullptr));
    if (nocc <= 0 || nocc > nb) return fail(HFGPU_ERR_ARG, "hfgpu_scf_create: nocc out of range");
    s->h = h;
    s->nb = nb;
    s->nocc = nocc;
    s->enuc = enuc;
    s->st = (cudaStream_t)hfgpu_stream(h);
    const size_t n2 = (size_t)nb * nb, bytes = n2 * sizeof(double);
    SCF_RC(acquire_linalg(s));
    for (auto& e : s->ev) SCF_CUDA(cudaEventCreate(&e));
    SCF_SOLVER(cusolverDnDsyevd_bufferSize(s->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, nullptr, nb,
                                           nullptr, &s->lwork));
    // every buffer of the job in one stream-ordered allocation (256-byte aligned pieces)
    const size_t ws = 4u << 20;  // cuBLAS gets its workspace here, so it never allocates later
    size_t off = 0;
    auto take = [&](size_t b) {
        const size_t o = off;
        off += (b + 255) / 256 * 256;
        return o;
    };
    double** mats[] = {&s->S, &s->H, &s->X, &s->P, &s->Pold, &s->F, &s->Fprev, &s->dP, &s->dF, &s->T1, &s->T2,
                       &s->Fob, &s->Cob};
    size_t o_mats[13], o_r[NDIIS], o_fo[NDIIS];
    for (int k = 0; k < 13; ++k) o_mats[k] = take(bytes);
    for (int k = 0; k < NDIIS; ++k) {
        o_r[k] = take(bytes);
        o_fo[k] = take(bytes);
    }
    const size_t o_w = take(nb * sizeof(double)), o_info = take(sizeof(int)), o_sc = take(sizeof(CycleScalars));
    const size_t o_aux = take((8 + 2 * (size_t)nb) * sizeof(double)), o_ws = take(ws);
    const size_t o_work = take((size_t)std::max(1, s->lwork) * sizeof(double));
    SCF_CUDA(hfgpu::pool_alloc(&s->arena, off, s->st));
    char* base = (char*)s->arena;
    for (int k = 0; k < 13; ++k) *mats[k] = (double*)(base + o_mats[k]);
    for (int k = 0; k < NDIIS; ++k) {
        s->R[k] = (double*)(base + o_r[k]);
        s->FO[k] = (double*)(base + o_fo[k]);
    }
    s->W = (double*)(base + o_w);
    s->info = (int*)(base + o_info);
    s->sc = (CycleScalars*)(base + o_sc);
    s->aux = (double*)(base + o_aux);
    s->blas_ws = base + o_ws;
    s->work = (double*)(base + o_work);
    s->bytes = off;
    SCF_BLAS(cublasSetWorkspace(s->blas, s->blas_ws, ws));
    SCF_CUDA(cudaMemcpyAsync(s->S, S, bytes, cudaMemcpyHostToDevice, s->st));
    SCF_CUDA(cudaMemcpyAsync(s->H, hcore, bytes, cudaMemcpyHostToDevice, s->st));
    // residual history starts at 1000 everywhere, as the reference's resido
    std::vector<double> big(n2, 1000.0);
    for (int k = 0; k < NDIIS; ++k) {
        SCF_CUDA(cudaMemcpyAsync(s->R[k], big.data(), bytes, cudaMemcpyHostToDevice, s->st));
        SCF_CUDA(cudaMemsetAsync(s->FO[k], 0, bytes, s->st));
    }
    SCF_CUDA(cudaStreamSynchronize(s->st));  // `big` leaves scope
    // S^-1/2 = U diag(1/sqrt(s)) U^T (direct_hartreefock.f90:22-29)
    SCF_RC(eigensolve(s, s->S));
    if (s->eigs[0] <= 0.0) return fail(HFGPU_ERR_ARG, "hfgpu_scf_create: S is not positive definite");
    k_scale_cols<<<(unsigned)((n2 + 255) / 256), 256, 0, s->st>>>(s->Cob, s->W, s->T1, nb);
    SCF_CUDA(cudaGetLastError());
    SCF_RC(gemm(s, false, true, 1.0, s->T1, s->Cob, 0.0, s->X));
    s->have_cob = false;
    if (p_guess) {  // atomic densities (direct_hartreefock.f90:50-59)
        SCF_CUDA(cudaMemcpyAsync(s->P, p_guess, bytes, cudaMemcpyHostToDevice, s->st));
        s->eelec = 0.0;
        s->uselevshft = false;
    } else {  // core Hamiltonian (:61-91)
        SCF_RC(gemm(s, false, false, 1.0, s->X, s->H, 0.0, s->T1));
        SCF_RC(gemm(s, false, true, 1.0, s->T1, s->X, 0.0, s->Fob));
        SCF_RC(eigensolve(s, s->Fob));
        SCF_RC(density_from_cob(s, s->P));
        double ph = 0.0;
        SCF_BLAS(cublasDdot(s->blas, (int)n2, s->P, 1, s->H, 1, &ph));
        s->eelec = ph;
        s->uselevshft = true;
    }
    SCF_RC(copy(s, s->Pold, s->P));
    SCF_CUDA(cudaStreamSynchronize(s->st));
    return HFGPU_OK;
}

int run(hfgpu_scf* s, const hfgpu_scf_params& prm, hfgpu_scf_result* res) {
    const int nb = s->nb;
    const size_t n2 = (size_t)nb * nb;
    hfgpu_handle* h = s->h;
    if (s->it == 0) {  // the protocol's start (direct_hartreefock.f90:31-38)
        for (int k = 0; k < NDIIS; ++k) s->slot[k] = k;
        for (int j = 0; j < NDIIS; ++j)
            for (int k = 0; k < NDIIS; ++k) s->B[j][k] = 1000.0 * 1000.0 * (double)n2;  // resido = 1000
        s->thresh = prm.lowthresh;
    }
    int* slot = s->slot;
    double* eo = s->eo;
    double (*B)[NDIIS] = s->B;
    bool& diis = s->diis;
    bool& fullfock = s->fullfock;
    bool& converged = s->converged;
    int& nusediis = s->nusediis;
    int& nfull = s->nfull;
    int& nfullb = s->nfullb;
    int& ndelta = s->ndelta;
    double& thresh = s->thresh;
    double& deltae = s->deltae;
    double& deltap = s->deltap;
    double eelec = s->eelec;
    const int grid = (int)std::min<size_t>((n2 + 255) / 256, 1024);
    while (!converged && s->it < prm.maxiter) {
        const int it = ++s->it;
        const double eeold = eelec;
        SCF_CUDA(cudaEventRecord(s->ev[0], s->st));
        SCF_RC(copy(s, s->F, s->H));
        if (fullfock && it == 1) {  // direct_hartreefock.f90:101-105 (fullfock stays set)
            SCF_RC(hfgpu_fock_build_initial_diag_device(h, s->F, s->P, thresh));
            SCF_RC(hfgpu_fock_build_non_diag_device(h, s->F, s->P, thresh, 0.0));
            nfull = 0;
            ++nfullb;
        } else if (fullfock) {      // :106-110
            SCF_RC(hfgpu_fock_build_device(h, s->F, s->P, thresh, thresh, 0.0));
            fullfock = false;
            nfull = 0;
            ++nfullb;
        } else {                    // :111-121, incremental on dP
            const double one = 1.0, mone = -1.0;
            SCF_BLAS(cublasDgeam(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, &one, s->P, nb, &mone, s->Pold, nb,
                                 s->dP, nb));
            SCF_CUDA(cudaMemsetAsync(s->dF, 0, n2 * sizeof(double), s->st));
            SCF_RC(hfgpu_fock_build_device(h, s->dF, s->dP, thresh, thresh * prm.fdifffac, prm.fp32_cutoff));
            SCF_BLAS(cublasDgeam(s->blas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, &one, s->Fprev, nb, &one, s->dF, nb, s->F,
                                 nb));
            if (++nfull == 15) fullfock = true;
            ++ndelta;
        }
        SCF_CUDA(cudaEventRecord(s->ev[1], s->st));
        SCF_RC(copy(s, s->Fprev, s->F));
        // fob = X F X^T; residual X^T (F P S - S P F) X, with S P F = (F P S)^T
        SCF_RC(gemm(s, false, false, 1.0, s->X, s->F, 0.0, s->T1));
        SCF_RC(gemm(s, false, true, 1.0, s->T1, s->X, 0.0, s->Fob));
        SCF_RC(gemm(s, false, false, 1.0, s->P, s->S, 0.0, s->T1));
        SCF_RC(gemm(s, false, false, 1.0, s->F, s->T1, 0.0, s->T2));
        {
            const double one = 1.0, mone = -1.0;
            SCF_BLAS(cublasDgeam(s->blas, CUBLAS_OP_N, CUBLAS_OP_T, nb, nb, &one, s->T2, nb, &mone, s->T2, nb, s->T1,
                                 nb));
        }
        // shift the histories: the oldest buffer takes the newest entry
        const int fresh = slot[NDIIS - 1];
        for (int k = NDIIS - 1; k > 0; --k) {
            slot[k] = slot[k - 1];
            eo[k] = eo[k - 1];
        }
        slot[0] = fresh;
        for (int j = NDIIS - 1; j > 0; --j)
            for (int k = NDIIS - 1; k > 0; --k) B[j][k] = B[j - 1][k - 1];
        SCF_RC(gemm(s, true, false, 1.0, s->X, s->T1, 0.0, s->T2));
        SCF_RC(gemm(s, false, false, 1.0, s->T2, s->X, 0.0, s->R[fresh]));
        SCF_RC(copy(s, s->FO[fresh], s->Fob));
        // the cycle's scalars
        SCF_CUDA(cudaMemsetAsync(s->sc, 0, sizeof(CycleScalars), s->st));
        {
            CycleArgs ca{};
            ca.P = s->P;
            ca.H = s->H;
            ca.F = s->F;
            ca.R = s->R[fresh];
            for (int k = 0; k < NDIIS; ++k) ca.Rj[k] = s->R[slot[k]];
            ca.Pold = s->Pold;
            ca.n = n2;
            k_cycle_scalars<<<grid, 256, 0, s->st>>>(ca, s->sc);
        }
        SCF_CUDA(cudaGetLastError());
        CycleScalars cs;
        SCF_CUDA(cudaMemcpyAsync(&cs, s->sc, sizeof(cs), cudaMemcpyDeviceToHost, s->st));
        SCF_CUDA(cudaStreamSynchronize(s->st));
        eelec = 0.5 * (cs.ph + cs.pf);  // :123-130
        deltae = eelec - eeold;
        double resmax;
        std::memcpy(&resmax, &cs.resmax, sizeof(double));
        std::memcpy(&deltap, &cs.dpmax, sizeof(double));
        for (int k = 0; k < NDIIS; ++k) B[0][k] = B[k][0] = cs.brow[k];
        eo[0] = eelec;
        if (it >= 2 && resmax < 0.3 && !diis) {  // :148-154
            diis = true;
            s->uselevshft = false;
        }
        if (it >= 7 && thresh > INTTHRESH && resmax < 0.005) {  // :155-160
            for (int k = 0; k < NDIIS; ++k) eo[k] = 2000.0;
            nusediis = 0;
            fullfock = true;
            s->uselevshft = false;
            thresh = INTTHRESH;
        }
        if (diis) {  // :161-199
            nusediis = std::min(nusediis + 1, NDIIS);
            if (nusediis > 1) {
                const int n = nusediis, m = n + 1;
                std::vector<double> A(m * m, 0.0), b(m, 0.0);
                for (int j = 0; j < n; ++j) {
                    for (int k = 0; k < n; ++k) A[j * m + k] = B[j][k];
                    A[j * m + n] = A[n * m + j] = -1.0;
                }
                b[n] = -1.0;
                int ii = 0;  // minloc(eo) over every history position
                for (int k = 1; k < NDIIS; ++k)
                    if (eo[k] < eo[ii]) ii = k;
                for (int j = 0; j < n; ++j)
                    if (j != ii) A[j * m + j] *= 1.05;
                double cmax = 0.0;
                const bool ok = small_solve(A, b, m);
                for (int j = 0; j < n && ok; ++j) cmax = std::max(cmax, std::fabs(b[j]));
                if (ok && cmax < 1.5) {
                    SCF_CUDA(cudaMemsetAsync(s->Fob, 0, n2 * sizeof(double), s->st));
                    for (int j = 0; j < n; ++j)
                        SCF_BLAS(cublasDaxpy(s->blas, (int)n2, &b[j], s->FO[slot[j]], 1, s->Fob, 1));
                } else {
                    nusediis = 0;
                }
            }
        }
        if (s->uselevshft && prm.levshft > 0.0 && s->have_cob && s->nocc < nb) {  // :200-203
            const double one = 1.0;
            const int nv = nb - s->nocc;
            SCF_BLAS(cublasDgemm(s->blas, CUBLAS_OP_N, CUBLAS_OP_T, nb, nb, nv, &prm.levshft,
                                 s->Cob + (size_t)s->nocc * nb, nb, s->Cob + (size_t)s->nocc * nb, nb, &one, s->Fob,
                                 nb));
        }
        // :204-205.  The eigenvectors are needed only while the level shift
        // acts on them; otherwise the density comes from purification and the
        // orbital energies are left for hfgpu_scf_get
        const bool vectors = s->uselevshft && prm.levshft > 0.0;
        if (vectors) SCF_RC(eigensolve(s, s->Fob));
        s->eigs_current = vectors;
        s->eelec = eelec;
        if (std::fabs(deltae) < prm.conve && deltap < prm.conv && it > 1) {  // :211-216
            converged = true;
            break;
        }
        SCF_RC(copy(s, s->Pold, s->P));
        SCF_CUDA(cudaEventRecord(s->ev[2], s->st));
        if (vectors) SCF_RC(density_from_cob(s, s->P));
        else SCF_RC(density_by_purification(s, s->Fob, s->P));
        SCF_CUDA(cudaEventRecord(s->ev[3], s->st));
        SCF_CUDA(cudaEventSynchronize(s->ev[3]));
        float mb = 0.f, md = 0.f;
        cudaEventElapsedTime(&mb, s->ev[0], s->ev[1]);
        cudaEventElapsedTime(&md, s->ev[2], s->ev[3]);
        s->ms_build += mb;
        s->ms_density += md;
    }
    SCF_CUDA(cudaStreamSynchronize(s->st));
    if (res) {
        res->energy = eelec + s->enuc;
        res->eelec = eelec;
        res->deltae = deltae;
        res->deltap = deltap;
        res->cycles = s->it;
        res->converged = converged ? 1 : 0;
        res->full_builds = nfullb;
        res->delta_builds = ndelta;
        res->sp2_steps = s->sp2_steps;
        res->ms_build = s->ms_build;
        res->ms_density = s->ms_density;
    }
    return HFGPU_OK;
}

}  // namespace

extern "C" {

void hfgpu_scf_defaults(hfgpu_scf_params* prm) {
    if (!prm) return;
    prm->maxiter = 25;
    prm->conv = 1e-5;
    prm->conve = 5e-8;
    prm->lowthresh = 5e-7;
    prm->fdifffac = 0.1;
    prm->fp32_cutoff = 0.0;
    prm->levshft = 0.0;
}

int hfgpu_scf_create(hfgpu_handle* h, int nocc, double enuc, const double* S, const double* hcore,
                     const double* p_guess, hfgpu_scf** out) {
    if (!h || !S || !hcore || !out) return fail(HFGPU_ERR_ARG, "hfgpu_scf_create: null argument");
    *out = nullptr;
    hfgpu_scf* s = new hfgpu_scf();
    const int rc = create(h, nocc, enuc, S, hcore, p_guess, s);
    if (rc) {
        release(s);
        return rc;
    }
    *out = s;
    return HFGPU_OK;
}

int hfgpu_scf_run(hfgpu_scf* s, const hfgpu_scf_params* prm, hfgpu_scf_result* res) {
    if (!s) return fail(HFGPU_ERR_ARG, "hfgpu_scf_run: null job");
    hfgpu_scf_params p;
    if (prm) p = *prm;
    else hfgpu_scf_defaults(&p);
    if (p.maxiter <= 0) return fail(HFGPU_ERR_ARG, "hfgpu_scf_run: maxiter must be positive");
    return run(s, p, res);
}

int hfgpu_scf_get(hfgpu_scf* s, double* p, double* f, double* eigs) {
    if (!s) return fail(HFGPU_ERR_ARG, "hfgpu_scf_get: null job");
    const size_t bytes = (size_t)s->nb * s->nb * sizeof(double);
    if (eigs && !s->eigs_current) {  // the last cycle's eigensolve, done on request
        int rc = eigensolve(s, s->Fob);
        if (rc) return rc;
        s->eigs_current = true;
    }
    if (p) SCF_CUDA(cudaMemcpyAsync(p, s->P, bytes, cudaMemcpyDeviceToHost, s->st));
    if (f) SCF_CUDA(cudaMemcpyAsync(f, s->Fprev, bytes, cudaMemcpyDeviceToHost, s->st));
    SCF_CUDA(cudaStreamSynchronize(s->st));
    if (eigs) std::copy(s->eigs.begin(), s->eigs.end(), eigs);
    return HFGPU_OK;
}

int hfgpu_scf_device_bytes(const hfgpu_scf* s, size_t* bytes) {
    if (!s || !bytes) return fail(HFGPU_ERR_ARG, "hfgpu_scf_device_bytes: null argument");
    *bytes = s->bytes;
    return HFGPU_OK;
}

int hfgpu_scf_destroy(hfgpu_scf* s) {
    if (s) release(s);
    return HFGPU_OK;
}

}  // extern "C"
