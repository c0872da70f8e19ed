"""Shared fixtures of the test-suite: molecules, shells and densities."""
from __future__ import annotations

import functools

import numpy as np

from hfcode_b200 import basis, molecules


@functools.lru_cache(maxsize=None)
def system(name: str):
    """(molecule, basis, shells, guess density).  A "_sp" suffix splits every
    L shell into S + pure P (same functions, pure-p quartet classes); "_mix"
    splits every other L shell, so S, P, D and L shells coexist."""
    if name.endswith("_sp") or name.endswith("_mix"):
        base, kind = name.rsplit("_", 1)
        mol, bas, sh, p0 = system(base)
        ls = [i for i in range(sh.nsh) if sh.shtyp[i] == basis.SHELL_L]
        which = None if kind == "sp" else set(ls[::2])
        return mol, bas, basis.split_l_shells(sh, which), p0
    return _system(name)


def _system(name: str):
    if name == "water":
        mol, bas = molecules.water(), basis.load_basis("STO-3G")
    elif name == "h2":  # s shells only: the SS|SS class alone
        mol, bas = basis.Molecule(["H", "H"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.74]])), \
            basis.load_basis("STO-3G")
    elif name == "ne":  # one centre: every quartet has AB = CD = PQ = 0 (Boys at T = 0)
        mol, bas = basis.Molecule(["Ne"], np.zeros((1, 3))), basis.load_basis("6-31G(d)")
    elif name == "benzene":
        mol, bas = molecules.benzene(), basis.load_basis("6-31G(d)")
    elif name == "c60":
        mol, bas = molecules.c60(), basis.load_basis("6-31G(d)")
    elif name.startswith("alkane"):
        mol, bas = molecules.alkane(int(name[6:])), basis.load_basis("6-31G(d)")
    elif name.startswith("wc"):
        k = int(name[2:])
        mol, bas = molecules.water_cluster(k, np.random.default_rng(20261203 + k)), basis.load_basis("6-31G(d)")
    else:
        raise KeyError(name)
    sh = basis.spread_basis(mol, bas)
    p0 = basis.density_superposition(mol, bas, sh.nb)
    return mol, bas, sh, p0


def perturbed_density(p0: np.ndarray, seed: int, scale: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = rng.normal(size=p0.shape) * scale
    return p0 + 0.5 * (d + d.T)
