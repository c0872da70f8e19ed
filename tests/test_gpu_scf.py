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
