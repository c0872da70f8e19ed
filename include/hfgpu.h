/*
 * hfgpu.h -- C ABI of the B200 direct-SCF Fock builder.
 *
 * Drop-in boundary for the reference's Fock builders.  Each entry point
 * replaces one external subroutine of brichjnh/hfcode that
 * direct_hartreefock.f90 calls (direct_hartreefock.f90:101-121); the
 * Fortran side binds them through an iso_c_binding interface module.
 *
 * Conventions shared by all entry points
 *   - f and p are caller-owned HOST arrays of nb x nb doubles, column-major
 *     (Fortran layout); p must be symmetric.
 *   - Semantics are accumulate: f += G(p), both triangles written, as the
 *     reference does (F = H + J - K/2 with the total density p = 2 C C^T).
 *   - Return 0 on success, non-zero on error; hfgpu_last_error() describes
 *     the last error of the calling thread.  The reference has no error
 *     convention (its subroutines `stop`); a Fortran shim `error stop`s on a
 *     non-zero return.
 *   - Calls on one handle are serialised on the handle's CUDA stream and are
 *     synchronous with respect to the host buffers they receive.  Different
 *     handles are independent.
 */
#ifndef HFGPU_H
#define HFGPU_H

#include "hfgpu_basis.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfgpu_handle hfgpu_handle;

/* Status codes. */
#define HFGPU_OK 0
#define HFGPU_ERR_ARG 1
#define HFGPU_ERR_CUDA 2
#define HFGPU_ERR_STATE 3
#define HFGPU_ERR_UNSUPPORTED 4
#define HFGPU_ERR_NOMEM 5

/* Replaces the one-time set-up the reference runs after reading the basis:
 * precalcs_kabs (precalc_kabs.f90:1-296: pair lists, primitive-pair data,
 * negab screen) and the Boys tables (index_functions.f90:171-226).
 * Uploads the shell data to the current CUDA device. */
int hfgpu_init(const hfgpu_basis* basis, hfgpu_handle** out);

/* Replaces fock_build_initial_diag(f,p,thr) (fock_build_initial_diag.f90:1-818):
 * (ab|ab) integrals of every shell pair, their Fock contributions with the
 * |e| > 1e-10 element skip, the Schwarz factors and their sorted, truncated
 * order (the reference's schwXX/orderXX/lastXX side effects,
 * fock_build_initial_diag.f90:51-52 ... 810-811).  Must precede the calls
 * below. */
int hfgpu_fock_build_initial_diag(hfgpu_handle* h, double* f, const double* p, double thr);

/* Replaces fock_build_diag(f,p,thr) (fock_build_diag.f90:1-692). */
int hfgpu_fock_build_diag(hfgpu_handle* h, double* f, const double* p, double thr);

/* Replaces fock_build_non_diag(f,p,thr) (fock_build_non_diag.f90:1-3412;
 * fock_build_non_diag_k.f90 is an identical copy). */
int hfgpu_fock_build_non_diag(hfgpu_handle* h, double* f, const double* p, double thr);

/* Replaces fock_build_non_diag_j_only(f,p,thr) (fock_build_non_diag_j.f90:1-2354):
 * Coulomb part only, screened by schw_ab*schw_cd*max(D_ab,D_cd). */
int hfgpu_fock_build_non_diag_j_only(hfgpu_handle* h, double* f, const double* p, double thr);

/* Mixed-precision off-diagonal build (no reference counterpart; the
 * reference is FP64 only, nrtype.f90:8-9).  Shell quartets whose screening
 * bound schw_ab*schw_cd*max(Dcoul,Dexch/4) falls below fp32_cutoff are
 * evaluated in FP32 (FP32 Boys, recurrences and contraction), the rest in
 * FP64; accumulation into f is FP64.  fp32_cutoff = 0 gives the FP64 build. */
int hfgpu_fock_build_non_diag_mixed(hfgpu_handle* h, double* f, const double* p, double thr,
                                    double fp32_cutoff);

/* Device-resident variant for callers that keep F and P in HBM: one full
 * build (fock_build_diag with thr_diag + fock_build_non_diag with
 * thr_non_diag, optionally mixed) on device pointers, enqueued on the
 * handle's stream; the host waits once, to read the per-class quartet
 * counts that size the launches.  f_dev += G(p_dev). */
int hfgpu_fock_build_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag,
                            double thr_non_diag, double fp32_cutoff);

/* Device-pointer forms of the cycle-1 calls (direct_hartreefock.f90:102-103):
 * f_dev += G_diag(p_dev) with the Schwarz pass (fock_build_initial_diag.f90),
 * and f_dev += G_non_diag(p_dev) alone (fock_build_non_diag.f90; FP32 below
 * fp32_cutoff when > 0).  nb x nb column-major device arrays; the initial
 * form synchronises the handle's stream to sort the Schwarz factors. */
int hfgpu_fock_build_initial_diag_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr);
int hfgpu_fock_build_non_diag_device(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr,
                                     double fp32_cutoff);

/* Batching form: the whole device build above recorded once as a CUDA graph
 * and replayed with one launch per build.  The 46 per-class loops of
 * fock_build_non_diag.f90 (and the diagonal builders) become one graph of
 * kernels on four concurrent branches; the per-class quartet counts stay on
 * the device, so a replay never returns to the host.  No counterpart in the
 * reference.
 *
 * hfgpu_graph_capture records f_dev += G(p_dev) with the given thresholds
 * and cutoff (replacing any earlier capture); the pointers are baked in, so
 * replays read whatever p_dev holds at that time.  It does not run the
 * build.  hfgpu_fock_build_initial_diag drops the capture (it re-sizes the
 * buffers the graph uses).  hfgpu_graph_launch enqueues one replay on the
 * handle's stream and returns; hfgpu_synchronize waits for the stream. */
int hfgpu_graph_capture(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag,
                        double thr_non_diag, double fp32_cutoff);
int hfgpu_graph_launch(hfgpu_handle* h);
int hfgpu_synchronize(hfgpu_handle* h);

/* The same replay behind the reference-style host interface: f += G(p) on
 * host arrays (fock_build_diag with thr_diag + fock_build_non_diag with
 * thr_non_diag, optionally mixed), through the handle's own device F and P
 * and a capture kept per (thresholds, cutoff) -- re-recorded when they
 * change.  One upload, one graph launch and one download per call. */
int hfgpu_fock_build_graph(hfgpu_handle* h, double* f, const double* p, double thr_diag, double thr_non_diag,
                           double fp32_cutoff);

/* One device build (as hfgpu_fock_build_device) enqueued on the caller's
 * CUDA stream without any host round trip: launches are sized by the class
 * capacities and the kernels read the survivor counts on the device, so a
 * caller may record it inside its own stream capture (a whole device-resident
 * SCF iteration as one graph).  No counterpart in the reference. */
int hfgpu_fock_build_device_on(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr_diag,
                               double thr_non_diag, double fp32_cutoff, void* stream);

/* Solves the small dense system A x = b (n <= 32; A row-major, overwritten;
 * x replaces b) on the device, enqueued on `stream`: the DIIS equations of a
 * device-resident SCF step (the role of wrapper_dsysv, wrapper_dsygv.f90:55-78).
 * *status_dev (if not NULL) is set to 1, or 0 for a singular matrix. */
int hfgpu_small_solve(double* a_dev, double* b_dev, int n, int* status_dev, void* stream);

/* Several SCF instances' captured builds as one graph launch: one child
 * graph per handle, no dependencies between them, so independent molecules
 * fill the GPU together.  Every handle must hold a capture (and appear
 * once); the batch copies the captures, stays valid while the handles live
 * and are not re-initialised, and is launched on any stream (NULL = the
 * legacy default stream). */
typedef struct hfgpu_batch hfgpu_batch;
int hfgpu_batch_create(hfgpu_handle* const* hs, int n, hfgpu_batch** out);
int hfgpu_batch_launch(hfgpu_batch* b, void* stream);
int hfgpu_batch_destroy(hfgpu_batch* b);

/* Number of basis functions / shells / shell pairs of the handle. */
int hfgpu_dims(const hfgpu_handle* h, int* nb, int* nsh, int* npairs);

/* Schwarz state left by hfgpu_fock_build_initial_diag: schw_sh (nsh x nsh,
 * row-major, symmetric) = sqrt(max |(ab|ab)|) per shell pair; last[10] =
 * the reference's lastXX per pair class in the order
 * ss, sp, sd, sl, pp, pd, pl, dd, dl, ll (index_sort.f90:95-119). */
int hfgpu_get_schwarz(const hfgpu_handle* h, double* schw_sh, int* last);

/* Statistics of the last off-diagonal build, per quartet class: arrays of
 * HFGPU_NCLASS entries.  The GPU pair types are SS LS LL DS DL DD PS LP PP DP
 * (larger shell first); classes 0..20 pair the first six types (i <= j, row
 * by row), classes 21..54 every pair of types that involves a pure p type
 * (i <= j, row by row, j >= 6).  Per class: screened-in shell quartets,
 * quartets that passed the max|e| post-screen, primitive quartets evaluated,
 * FP32 quartets (mixed form), and the kernel time in ms (0 unless timing is
 * enabled). */
#define HFGPU_NCLASS 55
int hfgpu_get_class_stats(const hfgpu_handle* h, long long* n_pass, long long* n_scattered,
                          long long* n_prim, long long* n_fp32, double* ms);

/* Kernels this handle has enqueued since hfgpu_init (graph and batch
 * replays count their captured kernels). */
int hfgpu_launch_count(const hfgpu_handle* h, long long* n);

/* Enable (1) or disable (0) per-class CUDA-event timing of the off-diagonal
 * kernels. */
int hfgpu_set_timing(hfgpu_handle* h, int on);

/* Upper bound in bytes of the staged classes' scratch (chunks of quartets
 * through the accumulator/output roles); set before
 * hfgpu_fock_build_initial_diag.  Default: HFGPU_SCRATCH_MB, else 24 GiB capped at
 * a sixth of the device's memory. */
int hfgpu_set_scratch_budget(hfgpu_handle* h, size_t bytes);

/* Device memory the handle holds, in bytes (pair data, screening tables,
 * quartet lists, scratch, F/P/G); used for admission by HBM footprint. */
int hfgpu_device_bytes(const hfgpu_handle* h, size_t* bytes);

/* The CUDA stream the handle enqueues on (a cudaStream_t). */
void* hfgpu_stream(hfgpu_handle* h);

/* Measures the FP64 and FP32 FMA throughput of the current device (GFLOP/s,
 * an FMA counted as 2) with an FMA-chain kernel; the denominators of the
 * Fock kernels' roofline.  No reference counterpart. */
int hfgpu_measure_fma_peak(double* fp64_gflops, double* fp32_gflops);

/* One-electron integrals S, T, V (nb x nb, symmetric) over the basis, with
 * the nuclei of charges[natom] at xyz[3*natom] (bohr).  Host code; replaces
 * cmpt1e.f90 / one_electron_terms.f90 (set-up, off the Fock-build path).
 * Any of S, T, V may be NULL. */
int hfgpu_one_electron(const hfgpu_basis* basis, int natom, const double* charges, const double* xyz,
                       double* S, double* T, double* V);

/* The same S, T, V computed on the current GPU (one thread per shell pair,
 * Obara-Saika recursions; host arrays in and out, temporary device buffers):
 * the GPU version of cmpt1e.f90 / one_electron_terms.f90:7-1059. */
int hfgpu_one_electron_gpu(const hfgpu_basis* basis, int natom, const double* charges, const double* xyz,
                           double* S, double* T, double* V);

/* fock_build_diag on device pointers for callers that cannot allocate GPU
 * memory at the call site -- for example code that runs where cudaMalloc is
 * not allowed, or that must not grow the device footprint after start-up.
 * No counterpart in the reference.  It allocates nothing: its scratch (the
 * accumulation buffer and the shell-pair density maxima) is a file-scope
 * __device__ array of 10,485,760 bytes (10.0 MiB) that every GPU loading the library holds until
 * exit, so nb <= 1024 and nsh <= 512 (larger sizes return HFGPU_ERR_ARG).
 * f_dev += G_diag(p_dev), enqueued on the handle's stream.  The handle must
 * come from hfgpu_init + hfgpu_fock_build_initial_diag, called earlier where
 * allocation is allowed.  The first call on a device looks up the scratch
 * address for that device; make that first call before any stream capture.
 * All calls share the one scratch array, so calls that overlap on the GPU
 * (other streams, other threads, other handles) race; serialise them. */
int hfgpu_fock_build_diag_static(hfgpu_handle* h, double* f_dev, const double* p_dev, double thr);

/* Releases all device memory of the handle (dealloc_integs.f90's role). */
int hfgpu_finalize(hfgpu_handle* h);

/* Text of the last error on the calling thread ("" if none). */
const char* hfgpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
