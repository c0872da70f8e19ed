"""Seeded geometry generators for the workloads the Fock builder is measured on.

All coordinates are in Angstrom (converted to bohr by ``basis.Molecule``).

* ``water``      -- O at the origin, O-H 0.9572 A, H-O-H 104.52 deg.
* ``benzene``    -- D6h ring, C-C 1.39 A, C-H 1.09 A.
* ``alkane(n)``  -- all-anti zig-zag CnH2n+2, C-C 1.53 A, C-H 1.09 A,
                    ideal tetrahedral angles, staggered methyl groups.
* ``c60``        -- ideal-Ih truncated icosahedron with 6-6 bonds 1.40 A and
                    5-6 bonds 1.45 A, built by cutting each icosahedron edge.
* ``water_cluster(k, rng)`` -- k rigid waters, seeded random orientations,
                    O-O >= 2.7 A by rejection sampling.

The reference ships stale-format inputs for some of these molecules; the
geometries here are generated from the stated bond lengths instead.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .basis import Molecule

TET = math.acos(-1.0 / 3.0)  # 109.4712 deg


def water(roh: float = 0.9572, angle_deg: float = 104.52) -> Molecule:
    h = math.radians(angle_deg) / 2.0
    xyz = np.array([[0.0, 0.0, 0.0],
                    [roh * math.sin(h), roh * math.cos(h), 0.0],
                    [-roh * math.sin(h), roh * math.cos(h), 0.0]])
    return Molecule(["O", "H", "H"], xyz)


def benzene(rcc: float = 1.39, rch: float = 1.09) -> Molecule:
    labels: List[str] = []
    xyz = []
    for k in range(6):
        t = math.pi / 3.0 * k
        labels.append("C"); xyz.append([rcc * math.cos(t), rcc * math.sin(t), 0.0])
    for k in range(6):
        t = math.pi / 3.0 * k
        r = rcc + rch
        labels.append("H"); xyz.append([r * math.cos(t), r * math.sin(t), 0.0])
    return Molecule(labels, np.array(xyz))


def _unit(v):
    return v / np.linalg.norm(v)


def alkane(n: int, rcc: float = 1.53, rch: float = 1.09) -> Molecule:
    """All-anti n-alkane CnH2n+2 in the xy plane (carbon zig-zag)."""
    if n < 1:
        raise ValueError("n >= 1")
    half = TET / 2.0
    dx, dy = rcc * math.sin(half), rcc * math.cos(half)

    def cpos(i):  # zig-zag carbon positions, extended to virtual i=-1 and i=n
        return np.array([i * dx, (i % 2) * dy, 0.0])

    labels = ["C"] * n
    xyz = [cpos(i) for i in range(n)]
    zhat = np.array([0.0, 0.0, 1.0])
    for i in range(n):
        c = cpos(i)
        left, right = cpos(i - 1), cpos(i + 1)
        nbrs = []
        if i > 0:
            nbrs.append(left)
        if i < n - 1:
            nbrs.append(right)
        # virtual neighbours continue the zig-zag; terminal carbons put an H there
        if i == 0:
            labels.append("H"); xyz.append(c + rch * _unit(left - c))
        if i == n - 1:
            labels.append("H"); xyz.append(c + rch * _unit(right - c))
        a, b = _unit(left - c), _unit(right - c)
        w = -_unit(a + b)
        for s in (1.0, -1.0):
            labels.append("H"); xyz.append(c + rch * (w * math.cos(half) + s * zhat * math.sin(half)))
    mol = Molecule(labels, np.array(xyz))
    if n == 1:
        # methane: regular tetrahedron
        v = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=float) / math.sqrt(3.0)
        mol = Molecule(["C", "H", "H", "H", "H"], np.vstack([[0, 0, 0], rch * v]))
    return mol


def c60(r66: float = 1.40, r56: float = 1.45) -> Molecule:
    """Truncated icosahedron: each icosahedron edge V_i->V_j carries two atoms
    at fractions t and 1-t, with t*a = r56 (pentagon side) and (1-2t)*a = r66."""
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    verts = []
    for s1 in (1, -1):
        for s2 in (1, -1):
            verts.append((0.0, s1 * 1.0, s2 * phi))
            verts.append((s1 * 1.0, s2 * phi, 0.0))
            verts.append((s1 * phi, 0.0, s2 * 1.0))
    v = np.array(verts)
    a = r66 + 2.0 * r56
    v *= a / 2.0  # unit icosahedron above has edge length 2
    t = r56 / a
    atoms = []
    for i in range(12):
        for j in range(12):
            if i != j and abs(np.linalg.norm(v[i] - v[j]) - a) < 1e-6:
                atoms.append(v[i] + t * (v[j] - v[i]))
    xyz = np.array(atoms)
    assert xyz.shape == (60, 3)
    return Molecule(["C"] * 60, xyz)


def water_cluster(k: int, rng: np.random.Generator, min_oo: float = 2.7, min_atom: float = 1.5,
                  box_per_mol: float = 3.3) -> Molecule:
    """k rigid waters at seeded random positions and orientations in a cube
    of ~box_per_mol A per molecule: O-O >= min_oo A by rejection sampling,
    and no two atoms of different waters closer than min_atom A."""
    mono = water().coords_ang
    side = box_per_mol * max(1.0, k ** (1.0 / 3.0))
    placed: List[np.ndarray] = []  # (3, 3) coordinates per water
    tries = 0
    while len(placed) < k:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place waters")
        c = rng.uniform(0.0, side, size=3) if placed else np.zeros(3)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        xyz = c + mono @ rot.T
        ok = True
        for other in placed:
            if np.linalg.norm(xyz[0] - other[0]) < min_oo or \
                    np.min(np.linalg.norm(xyz[:, None] - other[None], axis=-1)) < min_atom:
                ok = False
                break
        if ok:
            placed.append(xyz)
    labels = ["O", "H", "H"] * k
    return Molecule(labels, np.vstack(placed))


def by_name(name: str) -> Molecule:
    name = name.lower()
    if name == "water":
        return water()
    if name == "benzene":
        return benzene()
    if name == "c60":
        return c60()
    if name.startswith("c") and "h" in name:  # CnH2n+2, e.g. "c20h42"
        n = int(name[1:name.index("h")])
        return alkane(n)
    raise ValueError(name)
