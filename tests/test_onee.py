"""Host one-electron integrals (hfgpu_one_electron: Obara-Saika) against an
independent McMurchie-Davidson evaluation (tests/mdref.py) on s, p, l and d
shell pairs, including pairs on different atoms."""
import numpy as np
import pytest

from helpers import system
from hfcode_b200 import onee
import mdref


@pytest.mark.parametrize("name", ["water", "alkane1", "alkane2_mix"])
def test_one_electron_matches_mcmurchie_davidson(name):
    mol, _, sh, _ = system(name)
    S, T, V = onee.one_electron(mol, sh)
    atoms = list(zip(mol.charges, mol.coords))
    rng = np.random.default_rng(3)
    nfunc = {1: 1, 2: 3, 3: 5, 12: 4}
    pairs = {(a, b) for a in range(sh.nsh) for b in range(a + 1) if sh.shtyp[a] != sh.shtyp[b] or a == b}
    pairs = sorted(pairs)
    pick = [pairs[i] for i in rng.choice(len(pairs), size=min(12, len(pairs)), replace=False)]
    for a, b in pick:
        ref = mdref.shell_onee(sh, a, b, atoms)
        oa, ob = int(sh.aosh[a]), int(sh.aosh[b])
        na, nb = nfunc[int(sh.shtyp[a])], nfunc[int(sh.shtyp[b])]
        for got, r in zip((S, T, V), ref):
            blk = got[oa:oa + na, ob:ob + nb]
            assert np.max(np.abs(blk - r)) < 1e-10 * max(1.0, np.max(np.abs(r))), (name, a, b)
