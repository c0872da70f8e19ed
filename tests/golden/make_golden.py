"""Regenerates the golden fixtures of tests/golden from the CPU oracle alone.

    python tests/golden/make_golden.py [name ...]      (default: every system)

Everything here comes from oracle/ (liboracle.so and oracle/oscf.py): the
one-electron integrals, the Fock builds, the nuclear repulsion and the SCF
protocol.  Nothing from the product library (libhfgpu.so, hfcode_b200.scf,
hfcode_b200.onee) is called, so the GPU is compared with an independent
restatement of the reference.  The molecules, the shells and the
atomic-density guess are the inputs both sides share.

energies.json   converged RHF energies (direct_hartreefock protocol from the
                atomic-density guess): conve 1e-10 / conv 1e-7 for water/STO-3G,
                CH4 and benzene/6-31G(d); conve 1e-9 / conv 1e-6 for
                n-C20H42 and C60/6-31G(d).  Spherical d as the reference.
"_sp" systems   the same molecules with every L shell split into S + pure P
                (hfcode_b200.basis.split_l_shells): the pure-p classes.
fock_*.npz      small systems: F = fock_build_initial_diag + fock_build_non_diag
                at the atomic-density guess, thr 1e-10, F starting at zero.
fock_<big>.npz  n-C20H42 and C60: the lower triangles of F at the
                atomic-density guess ("sad") and at the oracle's
                core-Hamiltonian guess ("core", whose density P_core is stored
                too), with the oracle's screened-in and scattered quartet
                counts per reference class pair ([10, 10]: ss sp sd sl pp pd
                pl dd dl ll).
The reference publishes no outputs and cannot be compiled here, so these pin
the CUDA path against the oracle, not against hf.x itself.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from helpers import system  # noqa: E402
from oracle import oscf, pyoracle  # noqa: E402

SMALL = ["water", "alkane1", "benzene", "water_sp", "benzene_sp"]
BIG = {"c20h42": "alkane20", "c60": "c60"}


def tri(a):
    return a[np.tril_indices(a.shape[0])]


def energy(name, mol, sh, p0, conve, conv):
    t0 = time.time()
    r = oscf.OracleSCF(mol.charges, mol.coords, mol.nocc, sh).run(
        p_guess=p0, conve=conve, conv=conv, maxiter=80,
        log=lambda h: print(f"  {name} cycle {h['cycle']:2d} E {h['etot']:.10f} dE {h['deltae']:.2e} "
                            f"dP {h['deltap']:.2e}", flush=True))
    return {"energy": r["energy"], "cycles": r["cycles"], "converged": r["converged"], "nb": sh.nb,
            "conve": conve, "conv": conv, "seconds": round(time.time() - t0, 1)}


def small(name, energies):
    mol, bas, sh, p0 = system(name)
    orc = pyoracle.Oracle(sh)
    f = np.zeros((sh.nb, sh.nb))
    orc.fock_build_initial_diag(f, p0, 1e-10)
    orc.fock_build_non_diag(f, p0, 1e-10)
    np.savez_compressed(os.path.join(HERE, f"fock_{name}.npz"), F=f)
    energies[name] = energy(name, mol, sh, p0, 1e-10, 1e-7)


def big(name, energies):
    mol, bas, sh, p_sad = system(BIG[name])
    scf = oscf.OracleSCF(mol.charges, mol.coords, mol.nocc, sh)
    p_core = scf.core_density()
    out = {"P_core": tri(p_core)}
    for tag, p in (("sad", p_sad), ("core", p_core)):
        t0 = time.time()
        orc = pyoracle.Oracle(sh)
        f = np.zeros((sh.nb, sh.nb))
        orc.fock_build_initial_diag(f, p, 1e-10)
        orc.fock_build_non_diag(f, p, 1e-10)
        passed, scat = orc.counts()
        out[f"F_{tag}"] = tri(f)
        out[f"pass_{tag}"] = passed
        out[f"scat_{tag}"] = scat
        print(f"  {name} F at the {tag} guess: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"fock_{name}.npz"), **out)
    energies[name] = energy(name, mol, sh, p_sad, 1e-9, 1e-6)


def main(names):
    path = os.path.join(HERE, "energies.json")
    energies = json.load(open(path)) if os.path.exists(path) else {}
    for name in names:
        (big if name in BIG else small)(name, energies)
        print(name, energies[name], flush=True)
        with open(path, "w") as fh:
            json.dump(energies, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or SMALL + list(BIG))
