"""ctypes view of the C-ABI shell descriptor (include/hfgpu_basis.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from .basis import MAXPRIM, ShellSet

_i = ctypes.POINTER(ctypes.c_int)
_d = ctypes.POINTER(ctypes.c_double)


class HfgpuBasis(ctypes.Structure):
    _fields_ = [("nsh", ctypes.c_int), ("nb", ctypes.c_int), ("maxprim", ctypes.c_int),
                ("shtyp", _i), ("nzet", _i), ("atsh", _i), ("aosh", _i),
                ("xsh", _d), ("zeta", _d), ("djk", _d), ("djkl", _d)]


class BasisDescriptor:
    """Owns contiguous copies of a ShellSet's arrays and the struct pointing
    at them (the struct must not outlive this object)."""

    def __init__(self, sh: ShellSet):
        self.sh = sh
        self._keep = {
            "shtyp": np.ascontiguousarray(sh.shtyp, dtype=np.int32),
            "nzet": np.ascontiguousarray(sh.nzet, dtype=np.int32),
            "atsh": np.ascontiguousarray(sh.atsh, dtype=np.int32),
            "aosh": np.ascontiguousarray(sh.aosh, dtype=np.int32),
            "xsh": np.ascontiguousarray(sh.xsh, dtype=np.float64),
            "zeta": np.ascontiguousarray(sh.zeta, dtype=np.float64),
            "djk": np.ascontiguousarray(sh.djk, dtype=np.float64),
            "djkl": np.ascontiguousarray(sh.djkl, dtype=np.float64),
        }
        k = self._keep
        self.struct = HfgpuBasis(
            sh.nsh, sh.nb, MAXPRIM,
            k["shtyp"].ctypes.data_as(_i), k["nzet"].ctypes.data_as(_i),
            k["atsh"].ctypes.data_as(_i), k["aosh"].ctypes.data_as(_i),
            k["xsh"].ctypes.data_as(_d), k["zeta"].ctypes.data_as(_d),
            k["djk"].ctypes.data_as(_d), k["djkl"].ctypes.data_as(_d))

    @property
    def ref(self):
        return ctypes.byref(self.struct)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(_d)
