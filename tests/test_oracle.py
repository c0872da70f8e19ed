"""The CPU oracle against independent known answers (no GPU).

The reference ships no golden vectors, so the oracle is pinned by
mathematics: the Boys function against arbitrary precision, contracted ERIs
against an independent McMurchie-Davidson implementation, and the Fock
build against a brute-force J - K/2 from the full ERI tensor.
"""
import mpmath
import numpy as np
import pytest

import mdref
from helpers import system
from oracle import pyoracle

mpmath.mp.dps = 40


def exact_boys(m, T):
    if T == 0:
        return 1.0 / (2 * m + 1)
    return float(mpmath.gammainc(m + 0.5, 0, T) / (2 * mpmath.mpf(T) ** (m + 0.5)))


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 8])
def test_boys_below_28_is_exact(n):
    rng = np.random.default_rng(n)
    for T in list(rng.uniform(0, 28, 40)) + [0.0, 1e-16, 1.999, 2.0, 3.999, 4.0, 7.999, 8.0, 28.0]:
        f = pyoracle.boys(n, float(T))
        for m in range(n + 1):
            ex = exact_boys(m, float(T))
            assert abs(f[m] - ex) <= 5e-14 * ex, (n, m, T)


def test_boys_above_28_is_the_references_asymptotic_form():
    # boys.f90:24-27,134-139: no exponential term above x = 28
    for T in [28.5, 30.0, 45.0]:
        f = pyoracle.boys(8, T)
        g = mdref.boys_ref_longrange(8, T)
        assert np.allclose(f, g, rtol=1e-14, atol=0)


def test_oracle_eri_matches_mcmurchie_davidson():
    _, _, sh, _ = system("benzene")
    orc = pyoracle.Oracle(sh)
    rng = np.random.default_rng(7)
    d = [int(i) for i in np.where(sh.shtyp == 3)[0]]
    l_ = [int(i) for i in np.where(sh.shtyp == 12)[0]]
    s_ = [int(i) for i in np.where(sh.shtyp == 1)[0]]
    picks = [tuple(int(x) for x in rng.integers(0, sh.nsh, 4)) for _ in range(12)]
    picks += [(d[0], d[1], d[2], d[3]), (d[0], l_[0], s_[0], d[4]), (l_[0], l_[1], l_[2], l_[3]),
              (s_[0], s_[0], s_[1], s_[1]), (d[2], d[2], d[2], d[2])]
    for q in picks:
        e1 = orc.eri(*q)
        e2 = mdref.shell_eri(sh, *q, boysfn=mdref.boys_ref_longrange)
        assert np.max(np.abs(e1 - e2)) < 1e-13 * max(1.0, np.max(np.abs(e2))), q


@pytest.mark.parametrize("name", ["water", "alkane1"])
def test_oracle_fock_matches_bruteforce_jk(name):
    _, _, sh, _ = system(name)
    orc = pyoracle.Oracle(sh)
    nf = {1: 1, 2: 3, 3: 5, 12: 4}
    nb = sh.nb
    T = np.zeros((nb,) * 4)
    for a in range(sh.nsh):
        for b in range(sh.nsh):
            for c in range(sh.nsh):
                for d in range(sh.nsh):
                    n = [nf[int(sh.shtyp[s])] for s in (a, b, c, d)]
                    o = [int(sh.aosh[s]) for s in (a, b, c, d)]
                    T[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2], o[3]:o[3] + n[3]] = \
                        orc.eri(a, b, c, d).reshape(n)
    rng = np.random.default_rng(3)
    P = rng.normal(size=(nb, nb))
    P = P + P.T
    G = np.einsum("ijkl,kl->ij", T, P) - 0.5 * np.einsum("ikjl,kl->ij", T, P)
    F = np.zeros((nb, nb))
    orc.fock_build_initial_diag(F, P, 1e-14)
    orc.fock_build_non_diag(F, P, 1e-14)
    assert np.max(np.abs(F - G)) < 1e-9
    # J only
    J = np.einsum("ijkl,kl->ij", T, P)
    Fd = np.zeros((nb, nb))
    orc.fock_build_diag(Fd, P, 0.0)
    Fj = np.zeros((nb, nb))
    orc.fock_build_non_diag_j_only(Fj, P, 1e-14)
    # diag part holds J-K/2 of the (ab|ab) quartets; J-only covers the rest
    Jd = np.zeros((nb, nb))
    Fd2 = np.zeros((nb, nb))
    orc.fock_build_diag(Fd2, P, 0.0)
    assert np.allclose(Fd, Fd2)
    assert np.max(np.abs(Fj - (J - _diag_j(T, P, sh)))) < 1e-9


def _diag_j(T, P, sh):
    """Coulomb part restricted to quartets whose bra and ket shell pairs coincide."""
    nf = {1: 1, 2: 3, 3: 5, 12: 4}
    nb = sh.nb
    mask = np.zeros((nb,) * 4, dtype=bool)
    for a in range(sh.nsh):
        for b in range(sh.nsh):
            n = [nf[int(sh.shtyp[s])] for s in (a, b)]
            o = [int(sh.aosh[s]) for s in (a, b)]
            for (x, y) in ((a, b), (b, a)):
                ox, oy = int(sh.aosh[x]), int(sh.aosh[y])
                nx, ny = nf[int(sh.shtyp[x])], nf[int(sh.shtyp[y])]
                mask[o[0]:o[0] + n[0], o[1]:o[1] + n[1], ox:ox + nx, oy:oy + ny] = True
    return np.einsum("ijkl,kl->ij", np.where(mask, T, 0.0), P)


def test_maxdm_dl_block_follows_reference():
    # evaluate_maxdm.f90:82-89 reads rows d0..d3 and columns l0..l3 plus the
    # following function for d-l pairs
    _, _, sh, _ = system("alkane1")
    orc = pyoracle.Oracle(sh)
    nb = sh.nb
    P = np.zeros((nb, nb))
    d = int(np.where(sh.shtyp == 3)[0][0])
    l1 = int(np.where(sh.shtyp == 12)[0][0])
    P[sh.aosh[d] + 4, sh.aosh[l1]] = P[sh.aosh[l1], sh.aosh[d] + 4] = 5.0   # x2-y2 row: not read
    md = orc.maxdm(P)
    assert md[d, l1] == 0.0
    P[sh.aosh[d], sh.aosh[l1] + 4] = P[sh.aosh[l1] + 4, sh.aosh[d]] = 3.0   # function after l: read
    md = orc.maxdm(P)
    assert md[d, l1] == 3.0


@pytest.mark.parametrize("name", ["water", "alkane2_mix", "benzene"])
def test_oracle_one_electron_matches_mcmurchie_davidson(name):
    """The oracle's own S, T, V (cmpt1e.f90 / one_electron_terms.f90
    restated) against the independent McMurchie-Davidson evaluation on
    sampled shell pairs of every type combination present."""
    import mdref
    mol, _, sh, _ = system(name)
    S, T, V = pyoracle.Oracle(sh).one_electron(mol.charges, mol.coords)
    assert np.max(np.abs(S - S.T)) == 0 and np.max(np.abs(V - V.T)) == 0
    atoms = list(zip(mol.charges, mol.coords))
    nfunc = {1: 1, 2: 3, 3: 5, 12: 4}
    by_kind = {}
    for a in range(sh.nsh):
        for b in range(a + 1):
            by_kind.setdefault((int(sh.shtyp[a]), int(sh.shtyp[b]), a == b), []).append((a, b))
    rng = np.random.default_rng(7)
    for lst in by_kind.values():
        for k in rng.choice(len(lst), size=min(2, len(lst)), replace=False):
            a, b = lst[k]
            ref = mdref.shell_onee(sh, a, b, atoms)
            oa, ob = int(sh.aosh[a]), int(sh.aosh[b])
            na, nb = nfunc[int(sh.shtyp[a])], nfunc[int(sh.shtyp[b])]
            for got, r in zip((S, T, V), ref):
                blk = got[oa:oa + na, ob:ob + nb]
                assert np.max(np.abs(blk - r)) < 1e-10 * max(1.0, np.max(np.abs(r))), (name, a, b)


def test_oracle_scf_protocol_matches_golden():
    """The oracle's SCF (oracle/oscf.py) reproduces the golden water energy,
    which make_golden.py wrote with it (regression of the protocol)."""
    import json
    import os
    from oracle import oscf
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "energies.json")))["water"]
    mol, _, sh, p0 = system("water")
    r = oscf.OracleSCF(mol.charges, mol.coords, mol.nocc, sh).run(p_guess=p0, conve=1e-10, conv=1e-7)
    assert r["converged"] and abs(r["energy"] - gold["energy"]) < 1e-9
