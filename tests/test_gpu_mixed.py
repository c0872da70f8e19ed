"""The mixed FP32/FP64 form against the FP64 form, through the C ABI.

FP32 quartets carry ~1e-7 relative error; the cutoff bounds their size, so
the Fock matrix and the converged energy stay close to FP64.  Stated
tolerances: max|dF| <= 1e-5 for an all-FP32 off-diagonal build (every
quartet in FP32, a stress case well beyond any cutoff) on a perturbed density
of benzene, and |dE| <= 1e-6 Eh for the SCF with the mixed
incremental builds (the mixed form's accuracy target), which in practice lands far
below it."""
import json
import os

import numpy as np
import pytest

from helpers import perturbed_density, system
from hfcode_b200 import scf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.gpu
def test_all_fp32_build_is_close_to_fp64():
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system("benzene")
    fb = FockBuilder(sh)
    nb = sh.nb
    f0 = np.zeros((nb, nb))
    fb.fock_build_initial_diag(f0, p0, 1e-10)
    p = perturbed_density(p0, 3)
    f64, f32 = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_non_diag(f64, p, 1e-10)
    n64 = fb.class_stats()["pass"].sum()
    fb.fock_build_non_diag_mixed(f32, p, 1e-10, 1e30)
    st = fb.class_stats()
    assert st["fp32"].sum() == st["scattered"].sum() > 0   # every quartet in FP32
    assert st["pass"].sum() == n64
    d = np.max(np.abs(f32 - f64))
    assert 0 < d < 1e-5, d
    # cutoff 0 reproduces the FP64 build exactly in count and to round-off
    fz = np.zeros((nb, nb))
    fb.fock_build_non_diag_mixed(fz, p, 1e-10, 0.0)
    assert fb.class_stats()["fp32"].sum() == 0
    assert np.max(np.abs(fz - f64)) < 1e-12
    fb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,cutoff", [("benzene", 1e-7), ("benzene", 1e-4)])
def test_mixed_scf_energy(name, cutoff):
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(name)
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60, fp32_cutoff=cutoff)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold["energy"]) < 1e-6, (r.energy, gold["energy"])
