"""Basis-set ingestion and shell layout for the direct-SCF Fock builder.

Host-side mirror of the reference's input layer, restated in Python:

* ``read_basfile``  -- parse the reference's basis-file format
  (read_basfile.f90:1-96), including the optional atomic density blocks used
  by the superposition-of-atomic-densities guess (read_basfile.f90:71-91).
* ``normalize``     -- fold primitive normalisation into the contraction
  coefficients and renormalise the contracted shell (read_basfile.f90:100-179).
* ``spread_basis``  -- lay shells out atom-major, in basis-file order, and
  assign AO offsets; L shells store the p/s coefficient ratio
  (spread_basis.f90:1-182).

Shell type codes follow the reference (molprops.f90:75): s=1, p=2, d=3,
l(sp)=12.  d shells are spherical with 5 components in the order
z^2, xz, yz, xy, x^2-y^2 (index_functions.f90:147-168).

Units: coordinates are stored in bohr; the Angstrom->bohr factor is the
reference's 1.889725989 (read_infile.f90:6).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Sequence, Tuple

import numpy as np

BOHR = 1.889725989  # Angstrom -> bohr, read_infile.f90:6
MAXPRIM = 10        # molprops.f90:19

SHELL_S, SHELL_P, SHELL_D, SHELL_L = 1, 2, 3, 12
NFUNC = {SHELL_S: 1, SHELL_P: 3, SHELL_D: 5, SHELL_L: 4}

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

ELEMENTS = ["h", "he", "li", "be", "b", "c", "n", "o", "f", "ne",
            "na", "mg", "al", "si", "p", "s", "cl", "ar",
            "k", "ca", "sc", "ti", "v", "cr", "mn", "fe", "co", "ni", "cu", "zn",
            "ga", "ge", "as", "se", "br", "kr"]  # read_infile.f90:130-135


def atomic_number(label: str) -> int:
    """getnuccharge (read_infile.f90:122-149): element label -> Z."""
    lab = label.strip().lower()
    if lab not in ELEMENTS:
        raise ValueError(f"element not recognized: {label!r}")
    return ELEMENTS.index(lab) + 1


@dataclasses.dataclass
class ElementBasis:
    label: str
    shells: List[Tuple[int, np.ndarray, np.ndarray, np.ndarray]]  # (type, zeta, djk, djkl_abs)
    dmat: np.ndarray | None = None

    @property
    def nbf(self) -> int:
        return sum(NFUNC[t] for t, *_ in self.shells)


def normalize(zetas: np.ndarray, l: int, coefs: np.ndarray) -> np.ndarray:
    """Restates read_basfile.f90:100-179: returns d_jk = c_jk * N_prim,
    rescaled so the contracted shell has unit norm.  For d shells the
    primitive normalisation is that of the x^2 Cartesian component."""
    a = np.asarray(zetas, dtype=np.float64)
    g = np.asarray(coefs, dtype=np.float64).copy()
    pi = math.pi
    if l == 0:
        g *= (2.0 * a / pi) ** 0.75
    elif l == 1:
        g *= (2.0 / pi) ** 0.75 * 2.0 * a ** 1.25
    elif l == 2:
        g *= (2.0 / pi) ** 0.75 * 4.0 * a ** 1.75 / math.sqrt(3.0)
    pi32 = math.sqrt(pi ** 3)
    p = a[:, None] + a[None, :]
    gg = g[:, None] * g[None, :]
    if l == 0:
        nfac = np.sum(pi32 / np.sqrt(p ** 3) * gg)
    elif l == 1:
        nfac = np.sum(pi32 / (2.0 * p ** 2 * np.sqrt(p)) * gg)
    else:
        nfac = np.sum(pi32 * 3.0 / (4.0 * p ** 3 * np.sqrt(p)) * gg)
    return g / math.sqrt(nfac)


def _tokens(path: str):
    with open(path) as fh:
        for line in fh:
            yield line.split()


def read_basfile(path: str) -> Dict[str, ElementBasis]:
    """Parse a basis file in the reference format (read_basfile.f90:1-96).

    Header ``ELEMENTS n dmat``; per element: shell count, label, then per
    shell ``TYPE nprim [scale]`` followed by ``zeta c`` (or ``zeta c_s c_p``
    for L shells); ``****`` terminates an element.  With dmat=1 a
    ``DENSITY MATRICES`` section follows with one nbf x nbf block per element.
    """
    lines = [ln.split() for ln in open(path) if ln.strip()]
    pos = 0
    header = lines[pos]; pos += 1
    nel, dmat = int(header[1]), int(header[2])
    out: Dict[str, ElementBasis] = {}
    order: List[str] = []
    for _ in range(nel):
        nsh = int(lines[pos][0]); pos += 1
        label = lines[pos][0].lower(); pos += 1
        shells = []
        for _ in range(nsh):
            typ, nz = lines[pos][0].lower(), int(lines[pos][1]); pos += 1
            rows = [list(map(float, lines[pos + k])) for k in range(nz)]
            pos += nz
            z = np.array([r[0] for r in rows])
            if typ == "l":
                cs = normalize(z, 0, np.array([r[1] for r in rows]))
                cp = normalize(z, 1, np.array([r[2] for r in rows]))
                shells.append((SHELL_L, z, cs, cp))
            else:
                l = {"s": 0, "p": 1, "d": 2}[typ]
                c = normalize(z, l, np.array([r[1] for r in rows]))
                shells.append(({0: SHELL_S, 1: SHELL_P, 2: SHELL_D}[l], z, c, np.zeros_like(c)))
        assert lines[pos][0].startswith("****"), lines[pos]
        pos += 1
        out[label] = ElementBasis(label, shells)
        order.append(label)
    if dmat:
        pos += 1  # "DENSITY MATRICES"
        for label in order:
            pos += 1  # element label line
            eb = out[label]
            n = eb.nbf
            vals: List[float] = []
            while len(vals) < n * n:
                vals.extend(float(v) for v in lines[pos]); pos += 1
            eb.dmat = np.array(vals[: n * n]).reshape(n, n)
            assert lines[pos][0].startswith("****"), lines[pos]
            pos += 1
    return out


def basis_path(name: str) -> str:
    """Path of a bundled basis file by name ('6-31G(d)', 'STO-3G'), or the
    name itself when it is a path."""
    alias = {"6-31g(d)": "631Gd.dat", "631gd": "631Gd.dat", "6-31g*": "631Gd.dat",
             "sto-3g": "STO-3G.dat", "sto3g": "STO-3G.dat"}
    fn = alias.get(name.lower(), name)
    return fn if os.path.isabs(fn) or os.path.exists(fn) else os.path.join(DATA_DIR, fn)


def load_basis(name: str) -> Dict[str, ElementBasis]:
    """Load one of the bundled basis files by name ('6-31G(d)', 'STO-3G')
    or by path."""
    return read_basfile(basis_path(name))


@dataclasses.dataclass
class Molecule:
    labels: List[str]
    coords_ang: np.ndarray  # (natom, 3) Angstrom

    @property
    def coords(self) -> np.ndarray:
        return np.asarray(self.coords_ang, dtype=np.float64) * BOHR

    @property
    def charges(self) -> np.ndarray:
        return np.array([atomic_number(l) for l in self.labels], dtype=np.float64)

    @property
    def natom(self) -> int:
        return len(self.labels)

    def nuclear_repulsion(self) -> float:
        """nuclear_repulsion.f90:1-20."""
        x = self.coords
        z = self.charges
        e = 0.0
        for i in range(len(z)):
            for j in range(i + 1, len(z)):
                e += z[i] * z[j] / math.sqrt(float(np.sum((x[i] - x[j]) ** 2)))
        return e

    @property
    def nocc(self) -> int:
        return int(sum(atomic_number(l) for l in self.labels)) // 2


@dataclasses.dataclass
class ShellSet:
    """Flat per-shell arrays in the layout the C ABI consumes.

    ``zeta``, ``djk`` and ``djkl`` are (nsh, MAXPRIM); ``djkl`` holds the
    p/s coefficient *ratio* for L shells, exactly as spread_basis.f90:149-151
    stores it, and 0 elsewhere."""
    shtyp: np.ndarray   # int32 (nsh,)
    nzet: np.ndarray    # int32 (nsh,)
    atsh: np.ndarray    # int32 (nsh,) 0-based atom index
    aosh: np.ndarray    # int32 (nsh,) 0-based first AO
    xsh: np.ndarray     # float64 (nsh, 3) bohr
    zeta: np.ndarray    # float64 (nsh, MAXPRIM)
    djk: np.ndarray     # float64 (nsh, MAXPRIM)
    djkl: np.ndarray    # float64 (nsh, MAXPRIM)
    nb: int
    atcoords: np.ndarray  # (natom, 3) bohr
    nbfsat: np.ndarray    # int32 (natom,)

    @property
    def nsh(self) -> int:
        return int(self.shtyp.shape[0])

    def counts(self) -> Dict[str, int]:
        c = {k: int(np.sum(self.shtyp == v)) for k, v in
             (("s", SHELL_S), ("p", SHELL_P), ("d", SHELL_D), ("l", SHELL_L))}
        return c


def spread_basis(mol: Molecule, basis: Dict[str, ElementBasis]) -> ShellSet:
    """Restates spread_basis.f90:66-154: shells atom-major, in basis-file
    order; AO offsets assigned in the same walk.  Mixed P+D+L is rejected as
    the reference does (spread_basis.f90:174-177)."""
    shtyp, nzet, atsh, aosh, xsh, zeta, djk, djkl = [], [], [], [], [], [], [], []
    nbfsat = []
    iao = 0
    xyz = mol.coords
    for ia, lab in enumerate(mol.labels):
        eb = basis.get(lab.lower())
        if eb is None:
            raise ValueError(f"element {lab} not in basis")
        nbfsat.append(eb.nbf)
        for (t, z, cs, cp) in eb.shells:
            n = len(z)
            if n > MAXPRIM:
                raise ValueError("too many primitives")
            zz = np.zeros(MAXPRIM); zz[:n] = z
            dd = np.zeros(MAXPRIM); dd[:n] = cs
            ll = np.zeros(MAXPRIM)
            if t == SHELL_L:
                ll[:n] = cp / cs
            shtyp.append(t); nzet.append(n); atsh.append(ia); aosh.append(iao)
            xsh.append(xyz[ia]); zeta.append(zz); djk.append(dd); djkl.append(ll)
            iao += NFUNC[t]
    st = np.array(shtyp, dtype=np.int32)
    if np.any(st == SHELL_P) and np.any(st == SHELL_D) and np.any(st == SHELL_L):
        raise ValueError("Mixed P, D and L shells not supported")
    return ShellSet(st, np.array(nzet, np.int32), np.array(atsh, np.int32),
                    np.array(aosh, np.int32), np.array(xsh, np.float64).reshape(-1, 3),
                    np.array(zeta), np.array(djk), np.array(djkl), iao,
                    xyz.copy(), np.array(nbfsat, np.int32))


def split_l_shells(sh: ShellSet, which=None) -> ShellSet:
    """The same basis functions with L (sp) shells split into an S shell and
    a pure P shell of the same exponents (s coefficients djk, p coefficients
    djk * ratio), as bases such as 6-31G write them.  The AO order is
    unchanged: the S function keeps the L shell's first AO and the P shell
    follows it.  `which` selects the L shells to split (default: all)."""
    cols = {k: [] for k in ("shtyp", "nzet", "atsh", "aosh", "xsh", "zeta", "djk", "djkl")}
    for i in range(sh.nsh):
        row = dict(shtyp=int(sh.shtyp[i]), nzet=int(sh.nzet[i]), atsh=int(sh.atsh[i]), aosh=int(sh.aosh[i]),
                   xsh=sh.xsh[i], zeta=sh.zeta[i], djk=sh.djk[i], djkl=sh.djkl[i])
        if row["shtyp"] == SHELL_L and (which is None or i in which):
            srow = dict(row, shtyp=SHELL_S, djkl=np.zeros_like(sh.djkl[i]))
            prow = dict(row, shtyp=SHELL_P, aosh=row["aosh"] + 1, djk=sh.djk[i] * sh.djkl[i],
                        djkl=np.zeros_like(sh.djkl[i]))
            rows = [srow, prow]
        else:
            rows = [row]
        for r in rows:
            for k in cols:
                cols[k].append(r[k])
    return ShellSet(np.array(cols["shtyp"], np.int32), np.array(cols["nzet"], np.int32),
                    np.array(cols["atsh"], np.int32), np.array(cols["aosh"], np.int32),
                    np.array(cols["xsh"], np.float64).reshape(-1, 3), np.array(cols["zeta"]),
                    np.array(cols["djk"]), np.array(cols["djkl"]), sh.nb, sh.atcoords.copy(), sh.nbfsat.copy())


def density_superposition(mol: Molecule, basis: Dict[str, ElementBasis], nb: int) -> np.ndarray:
    """Guess density from atomic blocks (direct_hartreefock.f90:50-59)."""
    p = np.zeros((nb, nb))
    k = 0
    for lab in mol.labels:
        eb = basis[lab.lower()]
        if eb.dmat is None:
            raise ValueError("basis file has no density matrices")
        n = eb.nbf
        p[k:k + n, k:k + n] = eb.dmat
        k += n
    return p
