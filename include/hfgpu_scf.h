/*
 * hfgpu_scf.h -- device-resident RHF step of the B200 Fock builder.
 *
 * The reference runs its SCF cycle on the host between Fock builds
 * (direct_hartreefock.f90:98-223): energy, commutator residual, DIIS over
 * up to eight past Fock matrices, the eigensolve of the orthogonalised Fock
 * matrix (wrapper_dsyev, LAPACK dsyev) and the new density.  Here a job's
 * whole state -- density, Fock matrices, DIIS histories, S^-1/2, core
 * Hamiltonian and the builder's screening tables -- stays in the GPU's
 * memory, and the cycle runs from C++ on the builder handle's stream:
 * the Fock builds of this library and cuBLAS products.  The reference's
 * eigensolve gives the new density from the nocc lowest eigenvectors of the
 * orthogonalised Fock matrix; here that projector is formed by second-order
 * spectral projection (SP2, matrix products only), and cuSOLVER's syevd
 * (dsyev's role) runs only where eigenvectors are needed: the
 * core-Hamiltonian guess, cycles with the level shift on, and the orbital
 * energies on request.  A few scalars per cycle come back to the host, where
 * the protocol's decisions are taken as the reference takes them.
 *
 * One job per builder handle (the job uses the handle's stream); jobs on
 * different handles run concurrently from different host threads.
 * Matrices passed in and out are nb x nb, column-major, HOST arrays.
 * Every call returns 0 on success, else an HFGPU_ERR_* status (hfgpu.h)
 * with hfgpu_last_error() describing it.
 */
#ifndef HFGPU_SCF_H
#define HFGPU_SCF_H

#include "hfgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfgpu_scf hfgpu_scf;

/* Protocol parameters; hfgpu_scf_defaults() fills the reference's values
 * (direct_hartreefock.f90:13,19: maxiter 25, conv 1e-5, conve 5e-8,
 * lowthresh 5e-7, fdifffac 0.1, ndiis 8, no level shift). */
typedef struct {
    int maxiter;
    double conv;        /* max |dP| for convergence */
    double conve;       /* |dE| for convergence (Eh) */
    double lowthresh;   /* integral threshold of the early cycles */
    double fdifffac;    /* non-diagonal threshold factor of incremental builds */
    double fp32_cutoff; /* > 0: mixed form in the incremental builds (FP32 below this bound) */
    double levshft;     /* > 0: level shift of the virtual orbitals while it is on (:200-203) */
} hfgpu_scf_params;

typedef struct {
    double energy;      /* E_elec + E_nuc of the last cycle (Eh) */
    double eelec;
    double deltae;      /* energy change of the last cycle */
    double deltap;      /* max |dP| of the last cycle */
    int cycles;
    int converged;
    int full_builds;    /* Fock builds with the full density */
    int delta_builds;   /* incremental (dP) builds */
    int sp2_steps;      /* purification steps, all cycles */
    double ms_build;    /* device time in the Fock builds, all cycles (CUDA events) */
    double ms_density;  /* device time forming densities (purification or eigensolve) */
} hfgpu_scf_result;

void hfgpu_scf_defaults(hfgpu_scf_params* prm);

/* A job on builder h (hfgpu_init, no initial diag yet): nocc doubly occupied
 * orbitals, nuclear repulsion enuc, overlap S and core Hamiltonian
 * hcore = T + V, and the guess density p_guess (NULL: the core-Hamiltonian
 * guess of direct_hartreefock.f90:61-91).  Copies everything to the device
 * and forms S^-1/2 there (:22-29). */
int hfgpu_scf_create(hfgpu_handle* h, int nocc, double enuc, const double* S, const double* hcore,
                     const double* p_guess, hfgpu_scf** out);

/* Runs the protocol until convergence or until the job has done maxiter
 * cycles in all: a later call continues where the previous one stopped (a
 * call with maxiter 1 runs cycle 1, the Schwarz pass included).  prm NULL:
 * the defaults.  res receives the state after the last cycle run. */
int hfgpu_scf_run(hfgpu_scf* s, const hfgpu_scf_params* prm, hfgpu_scf_result* res);

/* Host copies of the current density, of the last Fock matrix (the
 * reference's faobold) and of the last cycle's orbital energies (nb values,
 * ascending; solved on request when the cycle did not need eigenvectors).
 * Any pointer may be NULL. */
int hfgpu_scf_get(hfgpu_scf* s, double* p, double* f, double* eigs);

/* Device memory held by the job (not counting the builder handle). */
int hfgpu_scf_device_bytes(const hfgpu_scf* s, size_t* bytes);

int hfgpu_scf_destroy(hfgpu_scf* s);

#ifdef __cplusplus
}
#endif

#endif
