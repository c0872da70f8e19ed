"""The two large configurations against the oracle, through the C ABI:
n-C20H42/6-31G(d) (nb = 364) and C60/6-31G(d) (nb = 840, all 21 classes).

Fixtures (tests/golden/make_golden.py, oracle only):
* F = fock_build_initial_diag + fock_build_non_diag from F = 0 at the
  atomic-density guess and at the oracle's core-Hamiltonian guess (its P is
  stored), thr 1e-10: every element within 1e-10 (the FP64 contract), and the
  screened-in quartets per class equal to the oracle's;
* the converged FP64 RHF energy of the reference's protocol (conve 1e-9,
  conv 1e-6): the GPU SCF within 1e-8 Eh;
* the mixed form on n-C20H42 at FP32 cutoff 1e-7 (the configuration the
  mixed target is quoted on): |dE| <= 1e-6 Eh against the oracle's FP64
  energy, and max|dF| of one mixed incremental build against the oracle's
  FP64 build of the same dP, printed and bounded.
"""
import json
import os

import numpy as np
import pytest

from helpers import system
from hfcode_b200 import scf
from test_gpu_parity import REF2GPU, gpu_class

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FTOL = 1e-10
ETOL = 1e-8
SYSTEMS = {"c20h42": "alkane20", "c60": "c60"}


def untri(v, nb):
    a = np.zeros((nb, nb))
    a[np.tril_indices(nb)] = v
    return a + np.tril(a, -1).T


def counts_by_gpu_class(passed):
    from hfcode_b200.fock import NCLASS
    out = np.zeros(NCLASS, dtype=np.int64)
    for ca in range(10):
        for cb in range(10):
            if passed[ca, cb]:
                out[gpu_class(REF2GPU[ca], REF2GPU[cb])] += passed[ca, cb]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("guess", ["sad", "core"])
@pytest.mark.parametrize("name", ["c20h42", "c60"])
def test_large_fock_matches_oracle(name, guess):
    from hfcode_b200.fock import FockBuilder
    fx = np.load(os.path.join(GOLD, f"fock_{name}.npz"))
    _, _, sh, p_sad = system(SYSTEMS[name])
    nb = sh.nb
    p = p_sad if guess == "sad" else untri(fx["P_core"], nb)
    fb = FockBuilder(sh)
    f = np.zeros((nb, nb))
    fb.fock_build_initial_diag(f, p, 1e-10)
    fb.fock_build_non_diag(f, p, 1e-10)
    counts = fb.class_stats()["pass"]
    fb.close()
    ref = untri(fx[f"F_{guess}"], nb)
    err = float(np.max(np.abs(f - ref)))
    print(f"{name} {guess}: max|F_gpu - F_oracle| = {err:.2e} over {nb}x{nb}")
    assert err < FTOL
    assert np.array_equal(counts, counts_by_gpu_class(fx[f"pass_{guess}"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c20h42", "c60"])
def test_large_scf_energy_matches_oracle(name):
    from hfcode_b200 import onee
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(SYSTEMS[name])
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=gold["conve"], conv=gold["conv"], maxiter=80,
                               ints=onee.one_electron(mol, sh, gpu=True))
    fb.close()
    print(f"{name}: E_gpu = {r.energy:.10f}, E_oracle = {gold['energy']:.10f}, "
          f"|dE| = {abs(r.energy - gold['energy']):.2e} Eh")
    assert r.converged
    assert abs(r.energy - gold["energy"]) < ETOL


@pytest.mark.gpu
def test_c20h42_mixed_form():
    from hfcode_b200 import onee
    from hfcode_b200.fock import FockBuilder
    from oracle import pyoracle
    cutoff = 1e-7
    gold = json.load(open(os.path.join(GOLD, "energies.json")))["c20h42"]
    fx = np.load(os.path.join(GOLD, "fock_c20h42.npz"))
    mol, _, sh, p0 = system("alkane20")
    nb = sh.nb
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=gold["conve"], conv=gold["conv"], maxiter=80,
                               ints=onee.one_electron(mol, sh, gpu=True), fp32_cutoff=cutoff)
    de = abs(r.energy - gold["energy"])
    # one incremental build on a delta-P between the two guesses, mixed on the
    # GPU against the FP64 oracle
    dp = untri(fx["P_core"], nb) - p0
    fg, fo = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_non_diag_mixed(fg, dp, 1e-11, cutoff)
    st = fb.class_stats()
    fb.close()
    orc = pyoracle.Oracle(sh)
    orc.fock_build_initial_diag(np.zeros((nb, nb)), p0, 1e-10)
    orc.fock_build_non_diag(fo, dp, 1e-11)
    df = float(np.max(np.abs(fg - fo)))
    frac = float(st["fp32"].sum() / max(1, st["scattered"].sum()))
    print(f"c20h42 mixed (FP32 cutoff {cutoff:g}): |dE| = {de:.2e} Eh vs the oracle's FP64 energy; "
          f"incremental build: max|dF| = {df:.2e} vs the oracle's FP64 build, {frac:.2f} of quartets in FP32")
    assert r.converged
    assert de <= 1e-6
    assert st["fp32"].sum() > 0
    assert df < 1e-6


@pytest.mark.gpu
def test_c20h42_j_only_and_incremental_builds_match_oracle():
    """n-C20H42 against the oracle run here: the Coulomb-only build
    (fock_build_non_diag_j.f90) at the core-guess density, and an
    incremental build (direct_hartreefock.f90:111-121: fock_build_diag at
    thr, fock_build_non_diag at thr*0.1) on the difference of the two
    guesses; 1e-10 element-wise, equal screened-in counts."""
    from hfcode_b200.fock import FockBuilder
    from oracle import pyoracle
    fx = np.load(os.path.join(GOLD, "fock_c20h42.npz"))
    _, _, sh, p_sad = system("alkane20")
    nb = sh.nb
    p_core = untri(fx["P_core"], nb)
    fb, orc = FockBuilder(sh), pyoracle.Oracle(sh)
    for obj in (fb, orc):
        obj.fock_build_initial_diag(np.zeros((nb, nb)), p_sad, 1e-10)
    jg, jo = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_non_diag_j_only(jg, p_core, 1e-10)
    orc.fock_build_non_diag_j_only(jo, p_core, 1e-10)
    assert np.max(np.abs(jg - jo)) < FTOL
    dp = p_core - p_sad
    dg, do = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_diag(dg, dp, 1e-10)
    orc.fock_build_diag(do, dp, 1e-10)
    fb.fock_build_non_diag(dg, dp, 1e-11)
    orc.fock_build_non_diag(do, dp, 1e-11)
    counts = fb.class_stats()["pass"]
    fb.close()
    err = float(np.max(np.abs(dg - do)))
    print(f"c20h42 incremental build: max|dF_gpu - dF_oracle| = {err:.2e}")
    assert err < FTOL
    assert np.array_equal(counts, counts_by_gpu_class(orc.counts()[0]))
