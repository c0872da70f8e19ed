"""ctypes wrapper of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this.  The
product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from hfcode_b200.cabi import BasisDescriptor

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
CLASSES = ["ss", "sp", "sd", "sl", "pp", "pd", "pl", "dd", "dl", "ll"]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def _lib():
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    d = ctypes.POINTER(ctypes.c_double)
    i = ctypes.POINTER(ctypes.c_int)
    ll = ctypes.POINTER(ctypes.c_longlong)
    vp = ctypes.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [vp]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_boys.argtypes = [ctypes.c_int, ctypes.c_double, d]
    lib.orc_eri.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, d]
    lib.orc_eri.restype = ctypes.c_int
    for n in ("orc_fock_build_diag", "orc_fock_build_non_diag", "orc_fock_build_non_diag_j_only"):
        getattr(lib, n).argtypes = [vp, d, d, ctypes.c_double]
        getattr(lib, n).restype = ctypes.c_int
    lib.orc_fock_build_initial_diag.argtypes = [vp, d, d, ctypes.c_double]
    lib.orc_schwarz.argtypes = [vp, d, i]
    lib.orc_counts.argtypes = [vp, ll, ll]
    lib.orc_maxdm.argtypes = [vp, d, d]
    lib.orc_num_threads.restype = ctypes.c_int
    lib.orc_one_electron.argtypes = [vp, ctypes.c_int, d, d, d, d, d]
    lib.orc_fock_build_non_diag_sample.argtypes = [vp, d, d, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    lib.orc_fock_build_non_diag_sample.restype = ctypes.c_longlong
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _lib()
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def boys(n: int, x: float) -> np.ndarray:
    out = np.zeros(n + 1)
    lib().orc_boys(n, x, _dp(out))
    return out


class Oracle:
    """Reference-semantics Fock builder on the CPU.  F is nb x nb, and is
    updated in place (F += G(P)), like the reference's fock_build_* calls."""

    def __init__(self, shells):
        self.desc = BasisDescriptor(shells)
        self.nb = shells.nb
        self.nsh = shells.nsh
        self.h = lib().orc_create(self.desc.ref)

    def __del__(self):
        try:
            if self.h:
                lib().orc_destroy(self.h)
        except Exception:
            pass

    @staticmethod
    def _fp(f, p):
        assert f.shape == p.shape and f.dtype == np.float64 and p.dtype == np.float64
        assert f.flags["F_CONTIGUOUS"] or f.flags["C_CONTIGUOUS"]
        return _dp(f), _dp(np.ascontiguousarray(p))

    def fock_build_initial_diag(self, f, p, thr):
        pp = np.ascontiguousarray(p)
        lib().orc_fock_build_initial_diag(self.h, _dp(f), _dp(pp), thr)

    def fock_build_diag(self, f, p, thr):
        pp = np.ascontiguousarray(p)
        if lib().orc_fock_build_diag(self.h, _dp(f), _dp(pp), thr) != 0:
            raise RuntimeError("fock_build_diag before fock_build_initial_diag")

    def fock_build_non_diag(self, f, p, thr):
        pp = np.ascontiguousarray(p)
        if lib().orc_fock_build_non_diag(self.h, _dp(f), _dp(pp), thr) != 0:
            raise RuntimeError("fock_build_non_diag before fock_build_initial_diag")

    def fock_build_non_diag_j_only(self, f, p, thr):
        pp = np.ascontiguousarray(p)
        if lib().orc_fock_build_non_diag_j_only(self.h, _dp(f), _dp(pp), thr) != 0:
            raise RuntimeError("fock_build_non_diag_j_only before fock_build_initial_diag")

    def fock_build_non_diag_sample(self, f, p, thr, stride, offset=0):
        pp = np.ascontiguousarray(p)
        n = lib().orc_fock_build_non_diag_sample(self.h, _dp(f), _dp(pp), thr, stride, offset)
        if n < 0:
            raise RuntimeError("sample before fock_build_initial_diag")
        return int(n)

    def eri(self, s1, s2, s3, s4):
        out = np.zeros(625)
        n = lib().orc_eri(self.h, s1, s2, s3, s4, _dp(out))
        return out[:n].copy()

    def schwarz(self):
        s = np.zeros((self.nsh, self.nsh))
        last = (ctypes.c_int * 10)()
        lib().orc_schwarz(self.h, _dp(s), last)
        return s, dict(zip(CLASSES, list(last)))

    def counts(self):
        a = (ctypes.c_longlong * 100)()
        b = (ctypes.c_longlong * 100)()
        lib().orc_counts(self.h, a, b)
        return np.array(list(a)).reshape(10, 10), np.array(list(b)).reshape(10, 10)

    def one_electron(self, charges, coords):
        """S, T, V (nb x nb) for nuclei of the given charges at coords (bohr)."""
        z = np.ascontiguousarray(charges, dtype=np.float64)
        x = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        S, T, V = (np.zeros((self.nb, self.nb)) for _ in range(3))
        lib().orc_one_electron(self.h, len(z), _dp(z), _dp(x), _dp(S), _dp(T), _dp(V))
        return S, T, V

    def maxdm(self, p):
        out = np.zeros((self.nsh, self.nsh))
        lib().orc_maxdm(self.h, _dp(np.ascontiguousarray(p)), _dp(out))
        return out
