"""The C ABI from a plain C program (no Python, no torch types): a caller
compiled with gcc against include/ and linked to libhfgpu.so reads the
reference's benzene input and the 6-31G(d) basis through the native input
layer, gets the shell view hfgpu_init takes, the density guess and the error
path, checked against the Python readers (no GPU compute).  The GPU test
then runs fock_build_initial_diag + fock_build_non_diag from C with host
arrays, the way the reference's SCF driver calls its builders."""
import os
import subprocess

import numpy as np
import pytest

from hfcode_b200 import basis, fock, inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INP = os.path.join(ROOT, "tests", "golden", "inputs", "benzene.inp")

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "hfgpu.h"
#include "hfgpu_ingest.h"

int main(int argc, char** argv) {
    hfgpu_system* s = NULL;
    if (hfgpu_system_from_files(argv[1], argv[2], &s)) {
        printf("error %s\n", hfgpu_last_error());
        return 2;
    }
    hfgpu_system_info info;
    hfgpu_basis v;
    if (hfgpu_system_get_info(s, &info) || hfgpu_system_basis(s, &v)) return 3;
    double* p = (double*)calloc((size_t)info.nb * info.nb, sizeof(double));
    if (hfgpu_system_density_guess(s, p)) return 4;
    double tr = 0.0, djk = 0.0;
    for (int i = 0; i < info.nb; ++i) tr += p[(size_t)i * info.nb + i];
    for (int i = 0; i < v.nsh * v.maxprim; ++i) djk += v.djk[i];
    printf("natom %d nsh %d nb %d nocc %d enuc %.12f trace %.12f djk %.12f last_aosh %d\n", info.natom, v.nsh,
           v.nb, info.nocc, info.enuc, tr, djk, v.aosh[v.nsh - 1]);
    free(p);
    hfgpu_system_free(s);
    hfgpu_system* bad = NULL;
    if (hfgpu_system_from_files(argv[1], "/nonexistent.inp", &bad) == 0 || bad != NULL) return 5;
    printf("error-path %s\n", hfgpu_last_error());
    return 0;
}
"""


def test_c_program_reads_inputs_through_the_c_abi(tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(fock.LIBPATH)
    subprocess.check_call(["gcc", "-std=c99", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                           "-L", libdir, "-lhfgpu", "-Wl,-rpath," + libdir])
    out = subprocess.run([str(exe), basis.basis_path("6-31G(d)"), INP], capture_output=True, text=True, check=True)
    line, err = out.stdout.strip().splitlines()
    f = line.split()
    got = dict(zip(f[0::2], f[1::2]))
    mol, _ = inputs.read_infile(INP)
    bas = basis.load_basis("6-31G(d)")
    sh = basis.spread_basis(mol, bas)
    p = basis.density_superposition(mol, bas, sh.nb)
    assert int(got["natom"]) == 12 and int(got["nsh"]) == sh.nsh and int(got["nb"]) == sh.nb == 96
    assert int(got["nocc"]) == mol.nocc and int(got["last_aosh"]) == int(sh.aosh[-1])
    assert abs(float(got["enuc"]) - mol.nuclear_repulsion()) < 1e-9
    assert abs(float(got["trace"]) - np.trace(p)) < 1e-9
    assert abs(float(got["djk"]) - sh.djk.sum()) < 1e-9
    assert err.startswith("error-path hfgpu_system_from_files: cannot open")


BUILD_PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "hfgpu.h"
#include "hfgpu_ingest.h"

/* the calls direct_hartreefock.f90:101-103 makes, from C with host arrays */
int main(int argc, char** argv) {
    hfgpu_system* s = NULL;
    hfgpu_basis v;
    hfgpu_system_info info;
    hfgpu_handle* h = NULL;
    if (hfgpu_system_from_files(argv[1], argv[2], &s) || hfgpu_system_get_info(s, &info) ||
        hfgpu_system_basis(s, &v) || hfgpu_init(&v, &h)) {
        fprintf(stderr, "%s\n", hfgpu_last_error());
        return 2;
    }
    const size_t n = (size_t)info.nb * info.nb;
    double* p = (double*)calloc(n, sizeof(double));
    double* f = (double*)calloc(n, sizeof(double));
    hfgpu_system_density_guess(s, p);
    if (hfgpu_fock_build_initial_diag(h, f, p, 1e-10) || hfgpu_fock_build_non_diag(h, f, p, 1e-10)) {
        fprintf(stderr, "%s\n", hfgpu_last_error());
        return 3;
    }
    FILE* o = fopen(argv[3], "wb");
    fwrite(f, sizeof(double), n, o);
    fclose(o);
    hfgpu_finalize(h);
    hfgpu_system_free(s);
    free(p);
    free(f);
    return 0;
}
"""


@pytest.mark.gpu
def test_c_program_runs_the_build_through_the_c_abi(tmp_path):
    """The same from C on the GPU: fock_build_initial_diag + non_diag on the
    atomic-density guess of benzene, F written by the C program and
    compared with the CPU oracle on the same shells (1e-10)."""
    from oracle import pyoracle
    src = tmp_path / "build.c"
    src.write_text(BUILD_PROGRAM)
    exe = tmp_path / "build"
    libdir = os.path.dirname(fock.LIBPATH)
    subprocess.check_call(["gcc", "-std=c99", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                           "-L", libdir, "-lhfgpu", "-Wl,-rpath," + libdir])
    fout = tmp_path / "f.bin"
    subprocess.run([str(exe), basis.basis_path("6-31G(d)"), INP, str(fout)], check=True, timeout=300)
    mol, _ = inputs.read_infile(INP)
    bas = basis.load_basis("6-31G(d)")
    sh = basis.spread_basis(mol, bas)
    p = basis.density_superposition(mol, bas, sh.nb)
    fc = np.fromfile(str(fout), dtype=np.float64).reshape(sh.nb, sh.nb, order="F")
    orc = pyoracle.Oracle(sh)
    fo = np.zeros((sh.nb, sh.nb), order="F")
    orc.fock_build_initial_diag(fo, p, 1e-10)
    orc.fock_build_non_diag(fo, p, 1e-10)
    assert np.max(np.abs(fc - fo)) < 1e-10
