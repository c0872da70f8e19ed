"""One-electron integrals on the GPU (hfgpu_one_electron_gpu) against the
oracle's own S, T, V (cmpt1e.f90 / one_electron_terms.f90 restated in
oracle/oracle.cpp) element-wise for s, p, l and d shells up to C60, and
directly against the independent McMurchie-Davidson evaluation
(tests/mdref.py) on sampled shell pairs."""
import numpy as np
import pytest

from helpers import system
from hfcode_b200 import basis, molecules, onee
from oracle import pyoracle


def _system(name):
    if name == "c60":
        mol = molecules.c60()
        return mol, basis.spread_basis(mol, basis.load_basis("6-31G(d)"))
    mol, _, sh, _ = system(name)
    return mol, sh


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "benzene", "benzene_sp", "alkane2_mix", "c60"])
def test_gpu_one_electron_matches_oracle(name):
    mol, sh = _system(name)
    ref = pyoracle.Oracle(sh).one_electron(mol.charges, mol.coords)
    dev = onee.one_electron(mol, sh, gpu=True)
    for r, d in zip(ref, dev):
        scale = max(1.0, np.max(np.abs(r)))
        assert np.max(np.abs(r - d)) < 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "alkane2_mix", "benzene"])
def test_gpu_one_electron_matches_mcmurchie_davidson(name):
    import mdref
    mol, sh = _system(name)
    S, T, V = onee.one_electron(mol, sh, gpu=True)
    atoms = list(zip(mol.charges, mol.coords))
    nfunc = {1: 1, 2: 3, 3: 5, 12: 4}
    rng = np.random.default_rng(11)
    pairs = [(a, b) for a in range(sh.nsh) for b in range(a + 1)]
    for k in rng.choice(len(pairs), size=min(10, len(pairs)), replace=False):
        a, b = pairs[k]
        ref = mdref.shell_onee(sh, a, b, atoms)
        oa, ob = int(sh.aosh[a]), int(sh.aosh[b])
        na, nb = nfunc[int(sh.shtyp[a])], nfunc[int(sh.shtyp[b])]
        for got, r in zip((S, T, V), ref):
            blk = got[oa:oa + na, ob:ob + nb]
            assert np.max(np.abs(blk - r)) < 1e-10 * max(1.0, np.max(np.abs(r))), (name, a, b)
