"""Python view of the native input layer (include/hfgpu_ingest.h).

`load_system` reads a basis file and a molecule input (or atoms given in
memory) in C++ and returns the same objects the Python readers build --
Molecule, InputOptions, ShellSet and the atomic-density guess -- so either
path can feed FockBuilder.  The C++ reader restates read_infile.f90,
read_basfile.f90 (with normalize), spread_basis.f90, nuclear_repulsion.f90
and the guess of direct_hartreefock.f90:50-59.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import basis, fock
from .basis import MAXPRIM, Molecule, ShellSet
from .cabi import HfgpuBasis
from .inputs import InputOptions

EXPORTS = ["hfgpu_system_from_files", "hfgpu_system_from_atoms", "hfgpu_system_get_info",
           "hfgpu_system_basis", "hfgpu_system_atoms", "hfgpu_system_atom_nbf",
           "hfgpu_system_density_guess", "hfgpu_system_free"]


class SystemInfo(ctypes.Structure):
    _fields_ = [("natom", ctypes.c_int), ("nsh", ctypes.c_int), ("nb", ctypes.c_int), ("maxprim", ctypes.c_int),
                ("nelec", ctypes.c_int), ("nocc", ctypes.c_int), ("has_density", ctypes.c_int),
                ("enuc", ctypes.c_double), ("densup", ctypes.c_int), ("directscf", ctypes.c_int),
                ("levshft", ctypes.c_int), ("lshft", ctypes.c_double), ("uhf", ctypes.c_int), ("sz", ctypes.c_int),
                ("mp2", ctypes.c_int), ("ccsd", ctypes.c_int), ("huckel", ctypes.c_int),
                ("prtlevl", ctypes.c_int), ("ncore", ctypes.c_int)]


def _setup():
    lib = fock.lib()
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    lib.hfgpu_system_from_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(vp)]
    lib.hfgpu_system_from_atoms.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), dp,
                                            ctypes.POINTER(vp)]
    lib.hfgpu_system_get_info.argtypes = [vp, ctypes.POINTER(SystemInfo)]
    lib.hfgpu_system_basis.argtypes = [vp, vp]
    lib.hfgpu_system_atoms.argtypes = [vp, ip, dp]
    lib.hfgpu_system_atom_nbf.argtypes = [vp, ip]
    lib.hfgpu_system_density_guess.argtypes = [vp, dp]
    lib.hfgpu_system_free.argtypes = [vp]
    lib.hfgpu_system_free.restype = None
    return lib


_lib = _setup()


def _check(rc, what):
    if rc != 0:
        raise fock.HfgpuError(f"{what} failed (status {rc}): {_lib.hfgpu_last_error().decode(errors='replace')}")


@dataclasses.dataclass
class NativeSystem:
    mol: Molecule
    options: InputOptions
    shells: ShellSet
    p_guess: Optional[np.ndarray]  # None when the basis file has no density blocks
    enuc: float
    nocc: int


def load_system(basfile: str, infile: Optional[str] = None, labels: Optional[Sequence[str]] = None,
                coords_ang: Optional[np.ndarray] = None) -> NativeSystem:
    """Read and lay out a system with the C++ input layer: either from a
    molecule input file or from element labels and Angstrom coordinates."""
    h = ctypes.c_void_p()
    bas = basis.basis_path(basfile).encode()
    if infile is not None:
        _check(_lib.hfgpu_system_from_files(bas, infile.encode(), ctypes.byref(h)), "hfgpu_system_from_files")
    else:
        xyz = np.ascontiguousarray(coords_ang, dtype=np.float64).reshape(-1, 3)
        labs = (ctypes.c_char_p * len(labels))(*[l.encode() for l in labels])
        _check(_lib.hfgpu_system_from_atoms(bas, len(labels), labs, xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            ctypes.byref(h)), "hfgpu_system_from_atoms")
    try:
        info = SystemInfo()
        _check(_lib.hfgpu_system_get_info(h, ctypes.byref(info)), "hfgpu_system_get_info")
        v = HfgpuBasis()
        _check(_lib.hfgpu_system_basis(h, ctypes.byref(v)), "hfgpu_system_basis")
        nsh, nat = info.nsh, info.natom

        def ia(ptr, n):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(np.int32).copy()

        def da(ptr, shape):
            return np.ctypeslib.as_array(ptr, shape=shape).astype(np.float64).copy()

        z = np.zeros(nat, np.int32)
        xyz_b = np.zeros((nat, 3))
        _check(_lib.hfgpu_system_atoms(h, z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       xyz_b.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "hfgpu_system_atoms")
        nbfat = np.zeros(nat, np.int32)
        _check(_lib.hfgpu_system_atom_nbf(h, nbfat.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "hfgpu_system_atom_nbf")
        sh = ShellSet(ia(v.shtyp, nsh), ia(v.nzet, nsh), ia(v.atsh, nsh), ia(v.aosh, nsh),
                      da(v.xsh, (nsh, 3)), da(v.zeta, (nsh, MAXPRIM)), da(v.djk, (nsh, MAXPRIM)),
                      da(v.djkl, (nsh, MAXPRIM)), info.nb, xyz_b, nbfat)
        p = None
        if info.has_density:
            pf = np.zeros(info.nb * info.nb)
            _check(_lib.hfgpu_system_density_guess(h, pf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                   "hfgpu_system_density_guess")
            p = pf.reshape(info.nb, info.nb, order="F").copy()
        labels_out = [basis.ELEMENTS[k - 1].capitalize() for k in z]
        mol = Molecule(labels_out, xyz_b / basis.BOHR)
        opt = InputOptions(densup=bool(info.densup), directscf=bool(info.directscf), levshft=bool(info.levshft),
                           lshft=info.lshft, uhf=bool(info.uhf), sz=info.sz, mp2=bool(info.mp2),
                           ccsd=bool(info.ccsd), huckel=bool(info.huckel), prtlevl=info.prtlevl, ncore=info.ncore)
        return NativeSystem(mol, opt, sh, p, info.enuc, info.nocc)
    finally:
        _lib.hfgpu_system_free(h)
