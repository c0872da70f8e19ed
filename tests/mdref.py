"""Independent contracted-ERI reference by McMurchie-Davidson (test helper).

Written from the published Hermite-expansion formulas (McMurchie & Davidson,
J. Comput. Phys. 26, 218 (1978); Helgaker, Jorgensen & Olsen ch. 9), not from
the reference or from the product's generator, so it can pin both the CPU
oracle and the CUDA kernels.  Boys values come from mpmath or from an exact
quadrature-free series, selectable so that the reference's large-argument
approximation can be mirrored when needed.
"""
from __future__ import annotations

import math

import mpmath
import numpy as np

SHELL_S, SHELL_P, SHELL_D, SHELL_L = 1, 2, 3, 12
CART = {
    SHELL_S: [(0, 0, 0)],
    SHELL_P: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    SHELL_L: [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
    SHELL_D: [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)],
}
R3 = math.sqrt(3.0)
HARM = np.array([[-.5, 0, 0, -.5, 0, 1.0],
                 [0, 0, R3, 0, 0, 0],
                 [0, 0, 0, 0, R3, 0],
                 [0, R3, 0, 0, 0, 0],
                 [R3 / 2, 0, 0, -R3 / 2, 0, 0]])

mpmath.mp.dps = 30


def boys_exact(nmax: int, T: float) -> np.ndarray:
    out = np.zeros(nmax + 1)
    for m in range(nmax + 1):
        if T < 1e-15:
            out[m] = 1.0 / (2 * m + 1)
        else:
            out[m] = float(mpmath.gammainc(m + 0.5, 0, T) / (2 * mpmath.mpf(T) ** (m + 0.5)))
    return out


def boys_ref_longrange(nmax: int, T: float) -> np.ndarray:
    """Exact below 28; above 28 the asymptotic form with upward recursion and
    no exponential term, which is what the reference evaluates there
    (boys.f90:24-27,134-139)."""
    if T <= 28.0:
        return boys_exact(nmax, T)
    out = np.zeros(nmax + 1)
    out[0] = 0.5 * math.sqrt(math.pi / T)
    for i in range(1, nmax + 1):
        out[i] = out[i - 1] * (i - 0.5) / T
    return out


def _E(i, j, t, Qx, a, b):
    """Hermite expansion coefficient E^{ij}_t for 1D overlap (recursive)."""
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return math.exp(-q * Qx * Qx)
    if j == 0:
        return (1 / (2 * p)) * _E(i - 1, j, t - 1, Qx, a, b) - (q * Qx / a) * _E(i - 1, j, t, Qx, a, b) \
            + (t + 1) * _E(i - 1, j, t + 1, Qx, a, b)
    return (1 / (2 * p)) * _E(i, j - 1, t - 1, Qx, a, b) + (q * Qx / b) * _E(i, j - 1, t, Qx, a, b) \
        + (t + 1) * _E(i, j - 1, t + 1, Qx, a, b)


def _R(t, u, v, n, p, PCx, PCy, PCz, F, cache):
    key = (t, u, v, n)
    if key in cache:
        return cache[key]
    if t < 0 or u < 0 or v < 0:
        return 0.0
    if t == u == v == 0:
        val = (-2 * p) ** n * F[n]
    elif t > 0:
        val = (t - 1) * _R(t - 2, u, v, n + 1, p, PCx, PCy, PCz, F, cache) + PCx * _R(t - 1, u, v, n + 1, p, PCx, PCy, PCz, F, cache)
    elif u > 0:
        val = (u - 1) * _R(t, u - 2, v, n + 1, p, PCx, PCy, PCz, F, cache) + PCy * _R(t, u - 1, v, n + 1, p, PCx, PCy, PCz, F, cache)
    else:
        val = (v - 1) * _R(t, u, v - 2, n + 1, p, PCx, PCy, PCz, F, cache) + PCz * _R(t, u, v - 1, n + 1, p, PCx, PCy, PCz, F, cache)
    cache[key] = val
    return val


def prim_eri(la, lb, lc, ld, a, b, c, d, A, B, C, D, boysfn=boys_exact):
    """Primitive Cartesian (ab|cd) over unnormalised x^l y^m z^n e^{-a r^2}."""
    p, q = a + b, c + d
    P = (a * A + b * B) / p
    Q = (c * C + d * D) / q
    alpha = p * q / (p + q)
    PQ = P - Q
    L = sum(la) + sum(lb) + sum(lc) + sum(ld)
    F = boysfn(L, alpha * float(PQ @ PQ))
    cache = {}
    val = 0.0
    Eab = [[_E(la[x], lb[x], t, A[x] - B[x], a, b) for t in range(la[x] + lb[x] + 1)] for x in range(3)]
    Ecd = [[_E(lc[x], ld[x], t, C[x] - D[x], c, d) for t in range(lc[x] + ld[x] + 1)] for x in range(3)]
    for t in range(len(Eab[0])):
        for u in range(len(Eab[1])):
            for v in range(len(Eab[2])):
                e1 = Eab[0][t] * Eab[1][u] * Eab[2][v]
                if e1 == 0.0:
                    continue
                for tau in range(len(Ecd[0])):
                    for nu in range(len(Ecd[1])):
                        for phi in range(len(Ecd[2])):
                            e2 = Ecd[0][tau] * Ecd[1][nu] * Ecd[2][phi]
                            if e2 == 0.0:
                                continue
                            val += e1 * e2 * (-1) ** (tau + nu + phi) * _R(t + tau, u + nu, v + phi, 0, alpha,
                                                                           PQ[0], PQ[1], PQ[2], F, cache)
    return 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * val


def shell_eri(sh, s1, s2, s3, s4, boysfn=boys_exact, negab=True):
    """Contracted ERI block (s1 s2|s3 s4) for a hfcode_b200.basis.ShellSet,
    function order per shell as the reference (L: s,x,y,z; d: z2,xz,yz,xy,x2-y2).
    Applies the reference's primitive-pair screen when negab is set."""
    shells = [s1, s2, s3, s4]
    typ = [int(sh.shtyp[s]) for s in shells]
    X = [np.asarray(sh.xsh[s], dtype=float) for s in shells]
    carts = [CART[t] for t in typ]
    nc = [len(c) for c in carts]
    acc = np.zeros(nc)
    rt2pi54 = math.sqrt(2 * math.pi ** 2 * math.sqrt(math.pi))

    def prims(sa, sb):
        out = []
        r2 = float(np.sum((sh.xsh[sa] - sh.xsh[sb]) ** 2))
        for za in range(sh.nzet[sa]):
            for zb in range(sh.nzet[sb]):
                ea, eb = sh.zeta[sa, za], sh.zeta[sb, zb]
                p = ea + eb
                K = rt2pi54 * math.exp(-ea * eb / p * r2) / p * sh.djk[sa, za] * sh.djk[sb, zb]
                if negab and abs(K) * math.sqrt(1 / p) < 1e-12:
                    continue
                out.append((za, zb))
        return out

    for za, zb in prims(s1, s2):
        for zc, zd in prims(s3, s4):
            z = [za, zb, zc, zd]
            e = [sh.zeta[shells[k], z[k]] for k in range(4)]
            dcoef = [sh.djk[shells[k], z[k]] for k in range(4)]
            ratio = [sh.djkl[shells[k], z[k]] for k in range(4)]
            for i, ca in enumerate(carts[0]):
                for j, cb in enumerate(carts[1]):
                    for k, cc in enumerate(carts[2]):
                        for l, cd in enumerate(carts[3]):
                            w = 1.0
                            for kk, comp in enumerate((ca, cb, cc, cd)):
                                w *= dcoef[kk]
                                if typ[kk] == SHELL_L and sum(comp) == 1:
                                    w *= ratio[kk]
                            acc[i, j, k, l] += w * prim_eri(ca, cb, cc, cd, e[0], e[1], e[2], e[3],
                                                            X[0], X[1], X[2], X[3], boysfn)
    for ax, t in enumerate(typ):
        if t == SHELL_D:
            acc = np.moveaxis(np.tensordot(HARM, np.moveaxis(acc, ax, 0), axes=(1, 0)), 0, ax)
    return acc.reshape(-1)


def _prim_onee(la, lb, a, b, A, B, atoms):
    """Primitive Cartesian overlap, kinetic and nuclear attraction by the
    Hermite expansion (McMurchie-Davidson); atoms = [(Z, C), ...]."""
    p = a + b
    P = (a * A + b * B) / p

    def s1(i, j, x):
        return _E(i, j, 0, A[x] - B[x], a, b) * math.sqrt(math.pi / p) if i >= 0 and j >= 0 else 0.0

    S = s1(la[0], lb[0], 0) * s1(la[1], lb[1], 1) * s1(la[2], lb[2], 2)
    T = 0.0
    for x in range(3):
        o = [s1(la[y], lb[y], y) for y in range(3) if y != x]
        l = lb[x]
        d2 = l * (l - 1) * s1(la[x], l - 2, x) - 2 * b * (2 * l + 1) * s1(la[x], l, x) \
            + 4 * b * b * s1(la[x], l + 2, x)
        T += -0.5 * d2 * o[0] * o[1]
    V = 0.0
    L = sum(la) + sum(lb)
    for Z, C in atoms:
        PC = P - C
        F = boys_exact(L, p * float(PC @ PC))
        cache = {}
        acc = 0.0
        for t in range(la[0] + lb[0] + 1):
            for u in range(la[1] + lb[1] + 1):
                for v in range(la[2] + lb[2] + 1):
                    acc += _E(la[0], lb[0], t, A[0] - B[0], a, b) * _E(la[1], lb[1], u, A[1] - B[1], a, b) * \
                        _E(la[2], lb[2], v, A[2] - B[2], a, b) * _R(t, u, v, 0, p, PC[0], PC[1], PC[2], F, cache)
        V += -Z * 2 * math.pi / p * acc
    return S, T, V


def shell_onee(sh, s1, s2, atoms):
    """Contracted (S, T, V) blocks of shells s1, s2 (functions in the
    reference's order, spherical d), with the L-shell p/s ratio."""
    typ = [int(sh.shtyp[s1]), int(sh.shtyp[s2])]
    X = [np.asarray(sh.xsh[s], dtype=float) for s in (s1, s2)]
    carts = [CART[t] for t in typ]
    out = [np.zeros((len(carts[0]), len(carts[1]))) for _ in range(3)]
    for za in range(sh.nzet[s1]):
        for zb in range(sh.nzet[s2]):
            ea, eb = sh.zeta[s1, za], sh.zeta[s2, zb]
            for i, ca in enumerate(carts[0]):
                for j, cb in enumerate(carts[1]):
                    w = sh.djk[s1, za] * sh.djk[s2, zb]
                    if typ[0] == SHELL_L and sum(ca) == 1:
                        w *= sh.djkl[s1, za]
                    if typ[1] == SHELL_L and sum(cb) == 1:
                        w *= sh.djkl[s2, zb]
                    vals = _prim_onee(ca, cb, ea, eb, X[0], X[1], atoms)
                    for k in range(3):
                        out[k][i, j] += w * vals[k]
    res = []
    for blk in out:
        if typ[0] == SHELL_D:
            blk = HARM @ blk
        if typ[1] == SHELL_D:
            blk = blk @ HARM.T
        res.append(blk)
    return res
