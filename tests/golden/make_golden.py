"""Regenerates the golden fixtures of tests/golden from the CPU oracle.

    python tests/golden/make_golden.py

energies.json   converged RHF energies (direct_hartreefock protocol, conve 1e-10,
                conv 1e-7, atomic-density guess) of water/STO-3G, CH4 and
                benzene/6-31G(d), spherical d as the reference.
"_sp" systems   the same molecules with every L shell split into S + pure P
                (hfcode_b200.basis.split_l_shells): the pure-p classes.
fock_*.npz      F = fock_build_initial_diag + fock_build_non_diag at the
                atomic-density guess, thr 1e-10, F starting at zero.
The reference publishes no outputs, so these pin the oracle against itself
across changes (regression), not against the reference.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from helpers import system  # noqa: E402
from hfcode_b200 import scf  # noqa: E402
from oracle import pyoracle  # noqa: E402

SYSTEMS = ["water", "alkane1", "benzene", "water_sp", "benzene_sp"]


def main():
    energies = {}
    for name in SYSTEMS:
        mol, bas, sh, p0 = system(name)
        orc = pyoracle.Oracle(sh)
        f = np.zeros((sh.nb, sh.nb))
        orc.fock_build_initial_diag(f, p0, 1e-10)
        orc.fock_build_non_diag(f, p0, 1e-10)
        np.savez_compressed(os.path.join(HERE, f"fock_{name}.npz"), F=f)
        r = scf.direct_hartreefock(mol, sh, pyoracle.Oracle(sh), p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
        energies[name] = {"energy": r.energy, "cycles": r.cycles, "converged": r.converged, "nb": sh.nb}
        print(name, energies[name])
    with open(os.path.join(HERE, "energies.json"), "w") as fh:
        json.dump(energies, fh, indent=1)


if __name__ == "__main__":
    main()
