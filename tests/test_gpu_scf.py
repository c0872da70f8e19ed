"""Converged RHF energies with the CUDA Fock builder against the oracle's
(golden fixtures), through the C ABI: |dE| <= 1e-8 Eh with both sides
converged to 1e-10 Eh under the reference's SCF protocol."""
import json
import os

import pytest

from helpers import system
from hfcode_b200 import scf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ETOL = 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "alkane1", "benzene"])
def test_gpu_scf_energy_matches_oracle(name):
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(name)
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold["energy"]) < ETOL, (r.energy, gold["energy"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "benzene"])
def test_pure_p_basis_energy(name):
    """The same basis functions written as S + pure P shells instead of L
    shells (the pure-p quartet classes): the converged energy matches the
    oracle's for that basis (golden, 1e-8 Eh).  Against the L-shell energy
    it agrees only to ~2e-7 Eh: the reference's screens act per shell pair,
    so splitting the shells changes which sub-threshold quartets are dropped
    (the oracle shows the same shift)."""
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))
    mol, _, sh, p0 = system(name + "_sp")
    assert (sh.shtyp == 2).any() and not (sh.shtyp == 12).any()
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold[name + "_sp"]["energy"]) < ETOL, (r.energy, gold[name + "_sp"]["energy"])
    assert abs(r.energy - gold[name]["energy"]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2", "ne"])
def test_gpu_scf_small_edge_systems(name):
    """Two s shells only (H2) and one centre (Ne: every quartet has
    AB = CD = PQ = 0): the GPU SCF energy against the oracle's own SCF
    (oracle/oscf.py: oracle integrals and protocol), computed here (both
    small), to 1e-8 Eh."""
    from hfcode_b200.fock import FockBuilder
    from oracle import oscf
    mol, _, sh, p0 = system(name)
    ref = oscf.OracleSCF(mol.charges, mol.coords, mol.nocc, sh).run(p_guess=p0, conve=1e-10, conv=1e-7,
                                                                     maxiter=60)
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
    fb.close()
    assert r.converged and ref["converged"]
    assert abs(r.energy - ref["energy"]) < ETOL, (r.energy, ref["energy"])
