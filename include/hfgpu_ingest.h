/*
 * hfgpu_ingest.h -- native input layer of the Fock builder: reads the
 * reference's basis files and molecule inputs and lays the shells out in the
 * hfgpu_basis form that hfgpu_init consumes.  Host code only; no entry point
 * here touches the GPU.
 *
 * Replaces, for a C or Fortran caller that wants the shells without the
 * reference's own set-up code:
 *   read_infile.f90:1-120   molecule input (atoms, coordinates, options)
 *   read_basfile.f90:1-96   basis file, incl. the atomic density blocks
 *   read_basfile.f90:100-179 normalize (primitive + contracted norms)
 *   spread_basis.f90:66-182 shells atom-major in basis-file order, AO offsets,
 *                            L-shell p/s coefficient ratio, mixed P/D/L check
 *   nuclear_repulsion.f90   nuclear repulsion energy
 *   direct_hartreefock.f90:50-59 atomic-density superposition guess
 *
 * Conventions: coordinates in bohr after loading (Angstrom in the input,
 * factor 1.889725989 as read_infile.f90:6); matrices column-major nb x nb;
 * every function returns 0 on success and non-zero with hfgpu_last_error()
 * describing the failure.
 */
#ifndef HFGPU_INGEST_H
#define HFGPU_INGEST_H

#include "hfgpu_basis.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfgpu_system hfgpu_system;

/* Scalars of a loaded system and the input file's options
 * (read_infile.f90:12-61; options absent from the file keep these defaults:
 * directscf 1, everything else 0). */
typedef struct hfgpu_system_info {
    int natom;
    int nsh;
    int nb;
    int maxprim;
    int nelec;        /* sum of nuclear charges (neutral molecule) */
    int nocc;         /* nelec / 2 */
    int has_density;  /* the basis file carries atomic density blocks */
    double enuc;      /* nuclear repulsion, hartree */
    int densup;       /* USEDENSITYSUPGUESS */
    int directscf;    /* DIRECTSCF */
    int levshft;      /* LEVELSHIFT flag */
    double lshft;     /* LEVELSHIFT value */
    int uhf;          /* UHF flag */
    int sz;           /* UHF 2S */
    int mp2;
    int ccsd;
    int huckel;       /* older inputs: HUCKEL guess flag */
    int prtlevl;      /* PRINT */
    int ncore;
} hfgpu_system_info;

/* Loads a molecule input file and a basis file and spreads the basis over
 * the atoms.  The result owns all its arrays. */
int hfgpu_system_from_files(const char* basfile, const char* infile, hfgpu_system** out);

/* The same from atoms given in memory: natom element labels ("C", "h", ...)
 * and natom x 3 row-major coordinates in Angstrom. */
int hfgpu_system_from_atoms(const char* basfile, int natom, const char* const* labels,
                            const double* coords_ang, hfgpu_system** out);

int hfgpu_system_get_info(const hfgpu_system* s, hfgpu_system_info* info);

/* Fills `view` with pointers into the system's shell arrays; they stay
 * valid until hfgpu_system_free(s).  `view` can be passed to hfgpu_init. */
int hfgpu_system_basis(const hfgpu_system* s, hfgpu_basis* view);

/* Nuclear charges (natom) and coordinates in bohr (natom x 3, row-major);
 * either pointer may be NULL. */
int hfgpu_system_atoms(const hfgpu_system* s, int* charges, double* coords_bohr);

/* Number of basis functions on each atom (natom). */
int hfgpu_system_atom_nbf(const hfgpu_system* s, int* nbf);

/* Superposition-of-atomic-densities guess P (nb x nb, column-major):
 * each atom's density block from the basis file on the diagonal.  Fails if
 * the basis file has no density blocks. */
int hfgpu_system_density_guess(const hfgpu_system* s, double* p);

void hfgpu_system_free(hfgpu_system* s);

#ifdef __cplusplus
}
#endif

#endif
