"""The generated class code, compiled for the host, against the CPU oracle.

The per-class device functions (contracted ERI block per role, J/K scatter
per role) are straight-line arithmetic emitted by gen_eri.py.  Built here
with g++ and a few CUDA shims (tests/hostcheck/host_eri.cpp), they are
checked class by class against the oracle's ERIs and against the uniform
degeneracy-weighted scatter, without a GPU.
"""
import ctypes
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import system
from hfcode_b200.cabi import BasisDescriptor
from oracle import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "hfcode_b200", "csrc")
GEN = os.path.join(CSRC, "generated")
TYPES = {1: "S", 2: "P", 12: "L", 3: "D"}
NFUNC = {1: 1, 2: 3, 12: 4, 3: 5}


def _gen():
    import sys
    sys.path.insert(0, CSRC)
    import gen_eri
    sys.path.pop(0)
    return gen_eri


def _build():
    import sys
    sys.path.insert(0, CSRC)
    import gen_eri
    sys.path.pop(0)
    gen_eri.main(GEN)
    srcs = [os.path.join(ROOT, "tests", "hostcheck", "host_eri.cpp"), os.path.join(CSRC, "types.cuh"),
            os.path.join(CSRC, "pairs.hpp"), os.path.join(CSRC, "scatter.cuh")] + sorted(
        os.path.join(GEN, f) for f in os.listdir(GEN) if f.endswith((".cuh", ".inc")))
    h = hashlib.sha1()
    for s in srcs:
        h.update(open(s, "rb").read())
    out = os.path.join(tempfile.gettempdir(), f"hfgpu_hostcheck_{h.hexdigest()[:16]}.so")
    if not os.path.exists(out):
        subprocess.check_call(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w", "-I", CSRC, "-o", out + ".tmp",
                               srcs[0]])
        os.replace(out + ".tmp", out)
    lib = ctypes.CDLL(out)
    vp, d = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    i = ctypes.c_int
    lib.hc_create.restype = vp
    lib.hc_create.argtypes = [vp]
    lib.hc_eri.argtypes = [vp, i, i, i, i, i, i, i, d]
    lib.hc_scatter.argtypes = [vp, i, i, i, i, i, d, ctypes.c_double, d, d, i, i]
    lib.hc_scatter.restype = i
    lib.hc_boys.argtypes = [vp, i, ctypes.c_double, d]
    return lib, json.load(open(os.path.join(GEN, "class_flops.json")))


@pytest.fixture(scope="module")
def host():
    return _build()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def class_quartets(sh, rng, n=3):
    """Shell quartets of every generated class in GPU orientation."""
    g = _gen()
    by = {t: [int(i) for i in np.where(sh.shtyp == c)[0]] for c, t in TYPES.items()}
    out = {}
    for ci, (bi, ki) in enumerate(g.class_list()):
        A, B = g.PAIR_TYPES[bi]
        C, D = g.PAIR_TYPES[ki]
        qs = [tuple(int(rng.choice(by[x])) for x in (A, B, C, D)) for _ in range(n)]
        if bi == ki:  # one quartet with the same pair twice (the diagonal builders' case)
            q = qs[0]
            qs.append((q[0], q[1], q[0], q[1]))
        out[ci] = qs
    return out


def test_generated_eri_matches_oracle(host):
    lib, info = host
    _, _, sh, _ = system("alkane2_mix")  # S, P, D and L shells: every class
    desc = BasisDescriptor(sh)
    h = lib.hc_create(ctypes.addressof(desc.struct))
    orc = pyoracle.Oracle(sh)
    rng = np.random.default_rng(11)
    for ci, qs in class_quartets(sh, rng).items():
        L = info[str(ci)]["L"]
        for q in qs:
            ref = orc.eri(*q)
            out = np.zeros(625)
            lib.hc_eri(h, ci, L, *q, 0, _dp(out))
            got = out[:ref.size]
            scale = max(1.0, np.max(np.abs(ref)))
            assert np.max(np.abs(got - ref)) < 1e-12 * scale, (info[str(ci)]["name"], q)
            out32 = np.zeros(625)
            lib.hc_eri(h, ci, L, *q, 1, _dp(out32))
            assert np.max(np.abs(out32[:ref.size] - ref)) < 2e-5 * scale, (info[str(ci)]["name"], q)


def test_generated_scatter_matches_uniform_scatter(host):
    lib, info = host
    _, _, sh, _ = system("alkane2_mix")
    desc = BasisDescriptor(sh)
    h = lib.hc_create(ctypes.addressof(desc.struct))
    orc = pyoracle.Oracle(sh)
    nb = sh.nb
    rng = np.random.default_rng(12)
    P = rng.normal(size=(nb, nb))
    P = np.asfortranarray(P + P.T)
    checked = 0
    for ci, qs in class_quartets(sh, rng, n=2).items():
        for q in qs:
            e = orc.eri(*q)
            na, nb_, nc, nd = (NFUNC[int(sh.shtyp[s])] for s in q)
            E = e.reshape(na, nb_, nc, nd)
            for jonly in (0, 1):
                s = 0.25
                G = np.zeros((nb, nb), order="F")
                rc = lib.hc_scatter(h, ci, *q, _dp(np.ascontiguousarray(e)), s, _dp(P), _dp(G), nb, jonly)
                assert rc == 0
                o = [int(sh.aosh[x]) for x in q]
                R = np.zeros((nb, nb), order="F")
                sl = [slice(o[k], o[k] + n) for k, n in enumerate((na, nb_, nc, nd))]
                R[sl[0], sl[1]] += 2 * s * np.einsum("ijkl,kl->ij", E, P[sl[2], sl[3]])
                R[sl[2], sl[3]] += 2 * s * np.einsum("ijkl,ij->kl", E, P[sl[0], sl[1]])
                if not jonly:
                    R[sl[0], sl[2]] -= 0.5 * s * np.einsum("ijkl,jl->ik", E, P[sl[1], sl[3]])
                    R[sl[0], sl[3]] -= 0.5 * s * np.einsum("ijkl,jk->il", E, P[sl[1], sl[2]])
                    R[sl[1], sl[2]] -= 0.5 * s * np.einsum("ijkl,il->jk", E, P[sl[0], sl[3]])
                    R[sl[1], sl[3]] -= 0.5 * s * np.einsum("ijkl,ik->jl", E, P[sl[0], sl[2]])
                # G is indexed G[r + c*nb] like the column-major R
                assert np.max(np.abs(G - R)) < 1e-12 * max(1.0, np.max(np.abs(R))), (info[str(ci)]["name"], q)
                checked += 1
    assert checked > 0


def test_device_boys_matches_exact(host):
    """The kernels' Boys function (8-term Taylor on a 1/8 grid, downward
    recursion with exp(-T) from the table and a 10-term Taylor factor)
    against mpmath below T = 28, and the reference's asymptotic form above."""
    import mdref
    lib, _ = host
    _, _, sh, _ = system("water")
    desc = BasisDescriptor(sh)
    h = lib.hc_create(ctypes.addressof(desc.struct))
    rng = np.random.default_rng(5)
    Ts = np.concatenate([[0.0, 1e-9, 0.0625, 0.125, 7.9375, 27.99], rng.uniform(0, 28, 40), rng.uniform(28.01, 60, 8)])
    for M in range(9):
        for T in Ts:
            out = np.zeros(9)
            lib.hc_boys(h, M, float(T), _dp(out))
            ref = mdref.boys_ref_longrange(M, float(T))
            rel = np.max(np.abs(out[:M + 1] - ref) / np.abs(ref))
            assert rel < 5e-14, (M, T, rel)
