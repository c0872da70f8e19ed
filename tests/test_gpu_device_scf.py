"""Device-resident SCF (hfcode_b200.device_scf): the reference's protocol with
each cycle a CUDA graph and the density from SP2 purification instead of an
eigensolver.  Converged energies must match the golden values (the oracle's
host SCF) to 1e-8 Eh, replayed and eager alike.  Late in benzene's SCF the
incremental builds let the energy wander by a few 1e-9 Eh around the full
build's value (the host driver does the same), so the cycle at which
|dE| < 1e-10 first holds varies from run to run with the order of the FP64
atomic sums; the cycle limit leaves room for that."""
import json
import os

import pytest

from helpers import system

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.gpu
@pytest.mark.parametrize("name,graphs", [("water", True), ("alkane1", True), ("benzene", True),
                                         ("benzene", False), ("water_sp", True)])
def test_device_scf_matches_golden(name, graphs):
    from hfcode_b200.device_scf import DeviceSCF
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(name)
    fb = FockBuilder(sh)
    r = DeviceSCF(mol, sh, fb, graphs=graphs).run(p0, conve=1e-10, conv=1e-7, maxiter=150)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold["energy"]) < 1e-8, (r.energy, gold["energy"], r.cycles)


@pytest.mark.gpu
def test_device_scf_mixed_precision():
    """Mixed form in the incremental builds: within 1e-6 Eh of the FP64 energy."""
    from hfcode_b200.device_scf import DeviceSCF
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))["benzene"]
    mol, _, sh, p0 = system("benzene")
    fb = FockBuilder(sh)
    r = DeviceSCF(mol, sh, fb).run(p0, conve=1e-10, conv=1e-7, maxiter=150, fp32_cutoff=1e-5)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold["energy"]) < 1e-6
