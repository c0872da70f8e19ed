"""The C-ABI library loads and exports every entry point include/*.h declares
(no GPU compute is called here)."""
import ctypes
import os
import re

from hfcode_b200 import fock, ingest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            syms |= set(re.findall(r"\b(hfgpu_[a-z0-9_]+)\s*\(", txt))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(fock.LIBPATH)
    syms = declared_symbols()
    assert "hfgpu_fock_build_non_diag" in syms
    for s in sorted(syms):
        assert hasattr(lib, s), s


def test_python_binding_lists_all_exports():
    assert set(fock.EXPORTS) | set(ingest.EXPORTS) >= declared_symbols()


def test_init_rejects_bad_arguments_without_gpu_compute():
    lib = fock.lib()
    h = ctypes.c_void_p()
    rc = lib.hfgpu_init(None, ctypes.byref(h))
    assert rc == 1
    assert b"bad arguments" in lib.hfgpu_last_error()
