"""The oracle reproduces its committed golden fixtures (tests/golden)."""
import json
import os

import numpy as np
import pytest

from helpers import system
from hfcode_b200 import scf
from oracle import pyoracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["water", "alkane1", "benzene", "water_sp", "benzene_sp"])
def test_oracle_fock_matches_golden(name):
    _, _, sh, p0 = system(name)
    orc = pyoracle.Oracle(sh)
    f = np.zeros((sh.nb, sh.nb))
    orc.fock_build_initial_diag(f, p0, 1e-10)
    orc.fock_build_non_diag(f, p0, 1e-10)
    ref = np.load(os.path.join(GOLD, f"fock_{name}.npz"))["F"]
    assert np.max(np.abs(f - ref)) < 1e-12


@pytest.mark.parametrize("name", ["water", "alkane1", "water_sp"])
def test_oracle_scf_energy_matches_golden(name):
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(name)
    r = scf.direct_hartreefock(mol, sh, pyoracle.Oracle(sh), p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
    assert r.converged
    assert abs(r.energy - gold["energy"]) < 1e-9
