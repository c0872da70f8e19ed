"""One-electron integrals and the core-Hamiltonian guess density.

S, T, V come from the C ABI's host routine hfgpu_one_electron (restating
cmpt1e.f90 / one_electron_terms.f90).  ``core_density`` is the reference's
non-superposition guess (direct_hartreefock.f90:22-29, 61-74): orthogonalise
with S^-1/2, diagonalise S^-1/2 H S^-1/2 and occupy the lowest nocc orbitals.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .basis import Molecule, ShellSet
from .cabi import BasisDescriptor
from . import fock


def one_electron(mol: Molecule, sh: ShellSet, gpu: bool = False):
    """S, T, V over the shells: on the host (hfgpu_one_electron) or, with
    gpu=True, on the current GPU (hfgpu_one_electron_gpu)."""
    lib = fock.lib()
    d = ctypes.POINTER(ctypes.c_double)
    fn = lib.hfgpu_one_electron_gpu if gpu else lib.hfgpu_one_electron
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, d, d, d, d, d]
    desc = BasisDescriptor(sh)
    nb = sh.nb
    S, T, V = (np.zeros((nb, nb)) for _ in range(3))
    z = np.ascontiguousarray(mol.charges, dtype=np.float64)
    x = np.ascontiguousarray(mol.coords, dtype=np.float64)
    args = (ctypes.addressof(desc.struct), mol.natom, z.ctypes.data_as(d), x.ctypes.data_as(d),
            S.ctypes.data_as(d), T.ctypes.data_as(d), V.ctypes.data_as(d))
    rc = fn(*args)  # the GPU form allocates stream-ordered on its own stream: no lock needed
    if rc != 0:
        msg = lib.hfgpu_last_error().decode(errors="replace") if gpu else ""
        raise fock.HfgpuError(f"{fn.__name__} failed ({rc}) {msg}")
    return S, T, V


def s_minus_half(S: np.ndarray) -> np.ndarray:
    """S^-1/2 as the reference forms it (direct_hartreefock.f90:22-29)."""
    e, U = np.linalg.eigh(S)
    return (U / np.sqrt(e)) @ U.T


def core_density(mol: Molecule, sh: ShellSet, ints=None) -> np.ndarray:
    S, T, V = ints if ints is not None else one_electron(mol, sh)
    X = s_minus_half(S)
    e, C = np.linalg.eigh(X @ (T + V) @ X.T)
    C = X @ C
    occ = C[:, :mol.nocc]
    return 2.0 * occ @ occ.T
