"""Python binding of the B200 Fock builder's C ABI (include/hfgpu.h).

Mirrors the reference's Fock-builder interface: the same three entry points
with the same arguments and the same accumulate semantics (f += G(p)), as
called by direct_hartreefock.f90:101-121:

    fb = FockBuilder(shells)
    fb.fock_build_initial_diag(f, p, thr)   # cycle 1: Schwarz + diagonal pairs
    fb.fock_build_non_diag(f, p, thr)
    fb.fock_build_diag(f, p, thr)           # later cycles
    fb.fock_build_non_diag(f, p, thr)

There is no CPU fallback: importing this module fails if the CUDA library
has not been built, and every call raises if the GPU reports an error.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Dict, Optional

import numpy as np

from .basis import ShellSet
from .cabi import BasisDescriptor

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libhfgpu.so")

# GPU pair types and quartet classes in the order of include/hfgpu.h
# (HFGPU_NCLASS): the 21 classes over the {s, l, d} types, then every class
# with a pure-p type
PAIR_TYPES = ["SS", "LS", "LL", "DS", "DL", "DD", "PS", "LP", "PP", "DP"]
CLASS_NAMES = ([f"{PAIR_TYPES[i]}|{PAIR_TYPES[j]}" for i in range(6) for j in range(i, 6)] +
               [f"{PAIR_TYPES[i]}|{PAIR_TYPES[j]}" for i in range(10) for j in range(i, 10) if j >= 6])
NCLASS = len(CLASS_NAMES)
REF_CLASSES = ["ss", "sp", "sd", "sl", "pp", "pd", "pl", "dd", "dl", "ll"]


class HfgpuError(RuntimeError):
    pass


# A stream capture in global mode forbids device-synchronising calls
# (cudaFree, ...) in every thread.  The library allocates stream-ordered and
# records its own captures in thread-local mode, so its calls need no lock;
# callers that record their own graphs around library calls (device_scf)
# hold this lock while recording, for their own framework's sake.
DEVICE_LOCK = threading.RLock()


class ScfParams(ctypes.Structure):
    """hfgpu_scf_params (include/hfgpu_scf.h)."""
    _fields_ = [("maxiter", ctypes.c_int), ("conv", ctypes.c_double), ("conve", ctypes.c_double),
                ("lowthresh", ctypes.c_double), ("fdifffac", ctypes.c_double), ("fp32_cutoff", ctypes.c_double),
                ("levshft", ctypes.c_double)]


class ScfResult(ctypes.Structure):
    """hfgpu_scf_result (include/hfgpu_scf.h)."""
    _fields_ = [("energy", ctypes.c_double), ("eelec", ctypes.c_double), ("deltae", ctypes.c_double),
                ("deltap", ctypes.c_double), ("cycles", ctypes.c_int), ("converged", ctypes.c_int),
                ("full_builds", ctypes.c_int), ("delta_builds", ctypes.c_int), ("sp2_steps", ctypes.c_int),
                ("ms_build", ctypes.c_double), ("ms_density", ctypes.c_double)]


def _load():
    if not os.path.exists(LIBPATH):
        raise ImportError(f"hfcode_b200: CUDA library {LIBPATH} is missing; run __graft_entry__.build()")
    lib = ctypes.CDLL(LIBPATH)
    d = ctypes.POINTER(ctypes.c_double)
    i = ctypes.POINTER(ctypes.c_int)
    ll = ctypes.POINTER(ctypes.c_longlong)
    vp = ctypes.c_void_p
    lib.hfgpu_init.argtypes = [vp, ctypes.POINTER(vp)]
    for n in ("hfgpu_fock_build_initial_diag", "hfgpu_fock_build_diag", "hfgpu_fock_build_non_diag",
              "hfgpu_fock_build_non_diag_j_only"):
        getattr(lib, n).argtypes = [vp, d, d, ctypes.c_double]
    lib.hfgpu_fock_build_non_diag_mixed.argtypes = [vp, d, d, ctypes.c_double, ctypes.c_double]
    lib.hfgpu_fock_build_device.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.hfgpu_dims.argtypes = [vp, i, i, i]
    lib.hfgpu_get_schwarz.argtypes = [vp, d, i]
    lib.hfgpu_get_class_stats.argtypes = [vp, ll, ll, ll, ll, d]
    lib.hfgpu_set_timing.argtypes = [vp, ctypes.c_int]
    lib.hfgpu_stream.argtypes = [vp]
    lib.hfgpu_stream.restype = vp
    lib.hfgpu_finalize.argtypes = [vp]
    lib.hfgpu_last_error.restype = ctypes.c_char_p
    lib.hfgpu_measure_fma_peak.argtypes = [d, d]
    lib.hfgpu_fock_build_diag_static.argtypes = [vp, vp, vp, ctypes.c_double]
    lib.hfgpu_set_scratch_budget.argtypes = [vp, ctypes.c_size_t]
    lib.hfgpu_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    lib.hfgpu_graph_capture.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.hfgpu_graph_launch.argtypes = [vp]
    lib.hfgpu_synchronize.argtypes = [vp]
    lib.hfgpu_fock_build_device_on.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, vp]
    lib.hfgpu_small_solve.argtypes = [vp, vp, ctypes.c_int, vp, vp]
    lib.hfgpu_launch_count.argtypes = [vp, ll]
    lib.hfgpu_fock_build_graph.argtypes = [vp, d, d, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.hfgpu_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    lib.hfgpu_batch_launch.argtypes = [vp, vp]
    lib.hfgpu_batch_destroy.argtypes = [vp]
    lib.hfgpu_fock_build_initial_diag_device.argtypes = [vp, vp, vp, ctypes.c_double]
    lib.hfgpu_fock_build_non_diag_device.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double]
    lib.hfgpu_scf_defaults.argtypes = [ctypes.POINTER(ScfParams)]
    lib.hfgpu_scf_defaults.restype = None
    lib.hfgpu_scf_create.argtypes = [vp, ctypes.c_int, ctypes.c_double, d, d, d, ctypes.POINTER(vp)]
    lib.hfgpu_scf_run.argtypes = [vp, ctypes.POINTER(ScfParams), ctypes.POINTER(ScfResult)]
    lib.hfgpu_scf_get.argtypes = [vp, d, d, d]
    lib.hfgpu_scf_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    lib.hfgpu_scf_destroy.argtypes = [vp]
    return lib


_lib = _load()

EXPORTS = ["hfgpu_init", "hfgpu_fock_build_initial_diag", "hfgpu_fock_build_diag",
           "hfgpu_fock_build_non_diag", "hfgpu_fock_build_non_diag_j_only",
           "hfgpu_fock_build_non_diag_mixed", "hfgpu_fock_build_device", "hfgpu_dims",
           "hfgpu_get_schwarz", "hfgpu_get_class_stats", "hfgpu_set_timing", "hfgpu_stream",
           "hfgpu_finalize", "hfgpu_last_error", "hfgpu_measure_fma_peak",
           "hfgpu_fock_build_diag_static", "hfgpu_one_electron", "hfgpu_set_scratch_budget",
           "hfgpu_device_bytes", "hfgpu_graph_capture", "hfgpu_graph_launch", "hfgpu_synchronize",
           "hfgpu_fock_build_graph", "hfgpu_launch_count", "hfgpu_fock_build_device_on",
           "hfgpu_small_solve", "hfgpu_one_electron_gpu",
           "hfgpu_batch_create", "hfgpu_batch_launch", "hfgpu_batch_destroy",
           "hfgpu_fock_build_initial_diag_device", "hfgpu_fock_build_non_diag_device",
           "hfgpu_scf_defaults", "hfgpu_scf_create", "hfgpu_scf_run", "hfgpu_scf_get", "hfgpu_scf_device_bytes",
           "hfgpu_scf_destroy"]


def measure_fma_peak():
    """(FP64, FP32) FMA throughput of the current GPU in GFLOP/s."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(_lib.hfgpu_measure_fma_peak(ctypes.byref(a), ctypes.byref(b)), "measure_fma_peak")
    return a.value, b.value


def lib():
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        msg = _lib.hfgpu_last_error().decode(errors="replace")
        raise HfgpuError(f"{what} failed (status {rc}): {msg}")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class FockBuilder:
    """One SCF instance's resident Fock-build state on the current GPU."""

    def __init__(self, shells: ShellSet, scratch_budget: Optional[int] = None):
        self.shells = shells
        self.nb = shells.nb
        self.nsh = shells.nsh
        self._desc = BasisDescriptor(shells)
        h = ctypes.c_void_p()
        _check(_lib.hfgpu_init(ctypes.addressof(self._desc.struct), ctypes.byref(h)), "hfgpu_init")
        self.h = h
        if scratch_budget is not None:
            self.set_scratch_budget(scratch_budget)

    def close(self):
        if getattr(self, "h", None):
            _lib.hfgpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _fp(self, f, p):
        if f.shape != (self.nb, self.nb) or p.shape != (self.nb, self.nb):
            raise ValueError("f and p must be nb x nb")
        if f.dtype != np.float64 or not (f.flags["C_CONTIGUOUS"] or f.flags["F_CONTIGUOUS"]):
            raise ValueError("f must be a contiguous float64 array (updated in place)")
        pp = np.ascontiguousarray(p, dtype=np.float64)
        return _dp(f), _dp(pp), pp

    # --- the reference's entry points -------------------------------------
    def fock_build_initial_diag(self, f: np.ndarray, p: np.ndarray, thr: float):
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_initial_diag(self.h, fp, pp, float(thr)), "fock_build_initial_diag")

    def fock_build_diag(self, f: np.ndarray, p: np.ndarray, thr: float):
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_diag(self.h, fp, pp, float(thr)), "fock_build_diag")

    def fock_build_non_diag(self, f: np.ndarray, p: np.ndarray, thr: float):
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_non_diag(self.h, fp, pp, float(thr)), "fock_build_non_diag")

    def fock_build_non_diag_j_only(self, f: np.ndarray, p: np.ndarray, thr: float):
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_non_diag_j_only(self.h, fp, pp, float(thr)), "fock_build_non_diag_j_only")

    # --- additions --------------------------------------------------------
    def fock_build_non_diag_mixed(self, f: np.ndarray, p: np.ndarray, thr: float, fp32_cutoff: float):
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_non_diag_mixed(self.h, fp, pp, float(thr), float(fp32_cutoff)),
               "fock_build_non_diag_mixed")

    def fock_build_device(self, f_ptr: int, p_ptr: int, thr_diag: float, thr_non_diag: float,
                          fp32_cutoff: float = 0.0):
        """Full build on device pointers (e.g. torch tensors' data_ptr())."""
        _check(_lib.hfgpu_fock_build_device(self.h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(p_ptr),
                                            float(thr_diag), float(thr_non_diag), float(fp32_cutoff)),
               "fock_build_device")

    def fock_build_diag_static(self, f_ptr: int, p_ptr: int, thr: float):
        """fock_build_diag on device pointers using the library's static
        scratch (no device allocation; see include/hfgpu.h)."""
        _check(_lib.hfgpu_fock_build_diag_static(self.h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(p_ptr),
                                                 float(thr)), "fock_build_diag_static")

    def graph_capture(self, f_ptr: int, p_ptr: int, thr_diag: float, thr_non_diag: float,
                      fp32_cutoff: float = 0.0):
        """Records fock_build_device on these device pointers as a CUDA graph
        (replayed by graph_launch; nothing runs now)."""
        _check(_lib.hfgpu_graph_capture(self.h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(p_ptr), float(thr_diag),
                                        float(thr_non_diag), float(fp32_cutoff)), "graph_capture")

    def fock_build_graph(self, f: np.ndarray, p: np.ndarray, thr_diag: float, thr_non_diag: float,
                         fp32_cutoff: float = 0.0):
        """f += G(p): fock_build_diag(thr_diag) + fock_build_non_diag(thr_non_diag)
        (mixed with fp32_cutoff > 0) as one CUDA-graph replay, host arrays."""
        fp, pp, keep = self._fp(f, p)
        _check(_lib.hfgpu_fock_build_graph(self.h, fp, pp, float(thr_diag), float(thr_non_diag),
                                           float(fp32_cutoff)), "fock_build_graph")

    def fock_build_device_on(self, f_ptr: int, p_ptr: int, thr_diag: float, thr_non_diag: float,
                             fp32_cutoff: float, stream: int):
        """fock_build_device enqueued on `stream` with no host round trip
        (safe inside the caller's CUDA-graph capture)."""
        _check(_lib.hfgpu_fock_build_device_on(self.h, ctypes.c_void_p(f_ptr), ctypes.c_void_p(p_ptr),
                                               float(thr_diag), float(thr_non_diag), float(fp32_cutoff),
                                               ctypes.c_void_p(stream)), "fock_build_device_on")

    def graph_launch(self):
        """Enqueues one replay of the captured build on the handle's stream."""
        _check(_lib.hfgpu_graph_launch(self.h), "graph_launch")

    def synchronize(self):
        _check(_lib.hfgpu_synchronize(self.h), "synchronize")

    def set_scratch_budget(self, nbytes: int):
        _check(_lib.hfgpu_set_scratch_budget(self.h, int(nbytes)), "set_scratch_budget")

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        _check(_lib.hfgpu_device_bytes(self.h, ctypes.byref(b)), "device_bytes")
        return int(b.value)

    def launch_count(self) -> int:
        """Kernels enqueued by this handle so far (graph replays included)."""
        n = ctypes.c_longlong()
        _check(_lib.hfgpu_launch_count(self.h, ctypes.byref(n)), "launch_count")
        return int(n.value)

    def stream(self) -> int:
        return int(_lib.hfgpu_stream(self.h) or 0)

    def set_timing(self, on: bool):
        _check(_lib.hfgpu_set_timing(self.h, 1 if on else 0), "set_timing")

    def schwarz(self):
        s = np.zeros((self.nsh, self.nsh))
        last = (ctypes.c_int * 10)()
        _check(_lib.hfgpu_get_schwarz(self.h, _dp(s), last), "get_schwarz")
        return s, dict(zip(REF_CLASSES, list(last)))

    def class_stats(self) -> Dict[str, np.ndarray]:
        arrs = [(ctypes.c_longlong * NCLASS)() for _ in range(4)]
        ms = (ctypes.c_double * NCLASS)()
        _check(_lib.hfgpu_get_class_stats(self.h, *arrs, ms), "get_class_stats")
        keys = ["pass", "scattered", "prim", "fp32"]
        out = {k: np.array(list(a), dtype=np.int64) for k, a in zip(keys, arrs)}
        out["ms"] = np.array(list(ms))
        return out


class DeviceSCFJob:
    """One RHF job whose state stays on the GPU (include/hfgpu_scf.h): the
    reference's SCF protocol run by the library from C++ on the builder's
    stream, cuSOLVER's syevd in the role of dsyev.  `builder` is a fresh
    FockBuilder (no initial diag yet); S and hcore = T + V are host arrays;
    p_guess None means the core-Hamiltonian guess."""

    def __init__(self, builder: "FockBuilder", nocc: int, enuc: float, S: np.ndarray, hcore: np.ndarray,
                 p_guess: Optional[np.ndarray] = None):
        self.builder = builder  # keeps the handle alive
        self.nb = builder.nb
        Sc = np.ascontiguousarray(S, dtype=np.float64)
        Hc = np.ascontiguousarray(hcore, dtype=np.float64)
        Pc = None if p_guess is None else np.ascontiguousarray(p_guess, dtype=np.float64)
        out = ctypes.c_void_p()
        # the job's buffers come from the stream-ordered allocator on the
        # builder's stream, so no library-wide lock is needed here
        _check(_lib.hfgpu_scf_create(builder.h, int(nocc), float(enuc), _dp(Sc), _dp(Hc),
                                     _dp(Pc) if Pc is not None else None, ctypes.byref(out)), "scf_create")
        self.s = out

    def run(self, maxiter: int = 25, conv: float = 1e-5, conve: float = 5e-8, fp32_cutoff: float = 0.0,
            levshft: float = 0.0, lowthresh: float = 5e-7, fdifffac: float = 0.1) -> Dict[str, float]:
        """Cycles until convergence or `maxiter` cycles in all (a later call
        continues); returns the state after the last cycle."""
        prm = ScfParams(int(maxiter), float(conv), float(conve), float(lowthresh), float(fdifffac),
                        float(fp32_cutoff), float(levshft))
        res = ScfResult()
        _check(_lib.hfgpu_scf_run(self.s, ctypes.byref(prm), ctypes.byref(res)), "scf_run")
        return {k: getattr(res, k) for k, _ in ScfResult._fields_}

    def get(self):
        """(P, F, orbital energies of the last cycle) as host arrays."""
        p, f, e = np.zeros((self.nb, self.nb)), np.zeros((self.nb, self.nb)), np.zeros(self.nb)
        _check(_lib.hfgpu_scf_get(self.s, _dp(p), _dp(f), _dp(e)), "scf_get")
        return p, f, e

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        _check(_lib.hfgpu_scf_device_bytes(self.s, ctypes.byref(b)), "scf_device_bytes")
        return int(b.value)

    def close(self):
        if getattr(self, "s", None):
            _lib.hfgpu_scf_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Captured builds of several FockBuilders replayed as one graph launch."""

    def __init__(self, builders):
        self.builders = list(builders)  # keeps the handles alive
        arr = (ctypes.c_void_p * len(self.builders))(*[b.h.value for b in self.builders])
        out = ctypes.c_void_p()
        _check(_lib.hfgpu_batch_create(arr, len(self.builders), ctypes.byref(out)), "batch_create")
        self.b = out

    def launch(self, stream: int = 0):
        _check(_lib.hfgpu_batch_launch(self.b, ctypes.c_void_p(stream)), "batch_launch")

    def close(self):
        if getattr(self, "b", None):
            _lib.hfgpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def small_solve(a_ptr: int, b_ptr: int, n: int, status_ptr: int, stream: int):
    """Device solve of A x = b (n <= 32, A row-major, x into b) on `stream`."""
    _check(_lib.hfgpu_small_solve(ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr), int(n),
                                  ctypes.c_void_p(status_ptr), ctypes.c_void_p(stream)), "small_solve")
