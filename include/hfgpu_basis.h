/*
 * hfgpu_basis.h -- the shell descriptor shared by the B200 Fock builder and
 * its CPU oracle.
 *
 * It carries exactly the per-shell state the reference keeps in module
 * `molprops` and that its Fock builders read implicitly
 * (molprops.f90:70-104, filled by spread_basis.f90:66-154):
 *
 *   shtyp  shell type: 1 = s, 2 = p, 3 = d (5 spherical), 12 = l (sp)
 *   nzet   number of primitives (<= maxprim)
 *   atsh   0-based atom index of the shell centre
 *   aosh   0-based index of the shell's first basis function
 *   xsh    centre coordinates in bohr, nsh x 3, row-major
 *   zeta   exponents, nsh x maxprim, row-major
 *   djk    contraction coefficients with primitive normalisation folded in
 *          (read_basfile.f90:100-179); for l shells the s-part coefficient
 *   djkl   for l shells the ratio p-coefficient / s-coefficient per
 *          primitive (spread_basis.f90:149-151); ignored otherwise
 *
 * All pointers are host memory owned by the caller and are only read during
 * the call that receives them.
 */
#ifndef HFGPU_BASIS_H
#define HFGPU_BASIS_H

#ifdef __cplusplus
extern "C" {
#endif

#define HFGPU_SHELL_S 1
#define HFGPU_SHELL_P 2
#define HFGPU_SHELL_D 3
#define HFGPU_SHELL_L 12

typedef struct hfgpu_basis {
    int nsh;
    int nb;
    int maxprim;
    const int* shtyp;
    const int* nzet;
    const int* atsh;
    const int* aosh;
    const double* xsh;
    const double* zeta;
    const double* djk;
    const double* djkl;
} hfgpu_basis;

#ifdef __cplusplus
}
#endif

#endif
