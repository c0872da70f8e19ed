"""The native (C++) input layer against the Python readers: the reference's
own input files in every header variant, both bundled basis files, atoms
given in memory (C60), the density guess, the error paths, and the CPU
oracle's Fock build on the shells each path lays out.  Integers and the
density blocks must be identical; normalised coefficients agree to a few
ulp (the sums run in another order)."""
import os

import numpy as np
import pytest

from hfcode_b200 import basis, ingest, inputs, molecules
from hfcode_b200.fock import HfgpuError

HERE = os.path.dirname(os.path.abspath(__file__))
INP = os.path.join(HERE, "golden", "inputs")
RTOL = 1e-14


def python_side(basname, infile=None, mol=None):
    if infile is not None:
        mol, opt = inputs.read_infile(infile)
    else:
        opt = None
    bas = basis.load_basis(basname)
    sh = basis.spread_basis(mol, bas)
    has_d = all(bas[l.lower()].dmat is not None for l in mol.labels)
    p = basis.density_superposition(mol, bas, sh.nb) if has_d else None
    return mol, opt, sh, p


def same_shells(a, b):
    assert a.nb == b.nb and a.nsh == b.nsh
    for k in ("shtyp", "nzet", "atsh", "aosh"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert np.array_equal(a.nbfsat, b.nbfsat)
    for k in ("xsh", "zeta", "djk", "djkl"):
        x, y = getattr(a, k), getattr(b, k)
        assert np.allclose(x, y, rtol=RTOL, atol=0.0), (k, np.max(np.abs(x - y)))
    assert np.allclose(a.atcoords, b.atcoords, rtol=RTOL, atol=1e-15)


@pytest.mark.parametrize("inp", ["h2oc", "h2ob", "c20h42", "benzene", "o"])
@pytest.mark.parametrize("basname", ["6-31G(d)", "STO-3G"])
def test_native_matches_python_on_reference_inputs(inp, basname):
    path = os.path.join(INP, inp + ".inp")
    ns = ingest.load_system(basname, infile=path)
    mol, opt, sh, p = python_side(basname, infile=path)
    same_shells(ns.shells, sh)
    assert ns.mol.labels == mol.labels
    assert ns.nocc == mol.nocc
    assert ns.enuc == pytest.approx(mol.nuclear_repulsion(), rel=RTOL)
    assert np.array_equal(ns.p_guess, p)
    for k in ("densup", "directscf", "levshft", "lshft", "uhf", "sz", "mp2", "ccsd", "huckel", "prtlevl", "ncore"):
        assert getattr(ns.options, k) == getattr(opt, k), k


def test_native_atoms_in_memory_c60():
    mol = molecules.c60()
    ns = ingest.load_system("6-31G(d)", labels=mol.labels, coords_ang=mol.coords_ang)
    _, _, sh, p = python_side("6-31G(d)", mol=mol)
    same_shells(ns.shells, sh)
    assert ns.shells.nb == 840 and ns.shells.counts() == {"s": 60, "p": 0, "d": 60, "l": 120}
    assert np.array_equal(ns.p_guess, p)
    assert ns.options.directscf and not ns.options.densup


def test_oracle_build_identical_on_either_layout():
    """The oracle's G(P) on the native shells equals the one on the Python
    shells (they describe the same functions to a few ulp)."""
    from oracle.pyoracle import Oracle
    path = os.path.join(INP, "h2oc.inp")
    ns = ingest.load_system("6-31G(d)", infile=path)
    _, _, sh, p = python_side("6-31G(d)", infile=path)
    out = []
    for s in (ns.shells, sh):
        o = Oracle(s)
        f = np.zeros((s.nb, s.nb))
        o.fock_build_initial_diag(f, p, 1e-10)
        o.fock_build_non_diag(f, p, 1e-10)
        out.append(f)
    assert np.max(np.abs(out[0] - out[1])) < 1e-13


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


BAS_NO_DMAT = """ELEMENTS 1 0
4
X
S 1 1.00
  1.5  1.0
P 1 1.00
  0.8  1.0
D 1 1.00
  0.6  1.0
L 2 1.00
  2.0  0.4  0.6
  0.5  0.7  0.5
****
"""


def test_basis_without_density_blocks_and_mixed_shells(tmp_path):
    bas = write(tmp_path, "x.dat", BAS_NO_DMAT.replace("X", "he"))
    with pytest.raises(HfgpuError, match="Mixed P, D and L"):
        ingest.load_system(bas, labels=["He"], coords_ang=np.zeros((1, 3)))
    with pytest.raises(ValueError, match="Mixed P, D and L"):
        basis.spread_basis(basis.Molecule(["He"], np.zeros((1, 3))), basis.read_basfile(bas))
    # without the P shell the same element loads; no density section
    txt = BAS_NO_DMAT.replace("X", "he").replace("4\nhe", "3\nhe").replace("P 1 1.00\n  0.8  1.0\n", "")
    bas2 = write(tmp_path, "y.dat", txt)
    ns = ingest.load_system(bas2, labels=["He", "he"], coords_ang=np.array([[0, 0, 0], [0, 0, 1.2]]))
    py = basis.spread_basis(basis.Molecule(["He", "He"], np.array([[0, 0, 0], [0, 0, 1.2]])),
                            basis.read_basfile(bas2))
    same_shells(ns.shells, py)
    assert ns.p_guess is None and ns.shells.nb == 2 * (1 + 5 + 4)


def test_fortran_exponents_and_blank_lines(tmp_path):
    """List-directed input: D exponents and blank lines between records."""
    txt = "ELEMENTS 1 0\n\n1\nH 0\nS 2 1.00\n  3.0D0  0.5d0\n\n  0.5  0.6\n****\n"
    ns = ingest.load_system(write(tmp_path, "h.dat", txt), labels=["H"], coords_ang=np.zeros((1, 3)))
    py = basis.spread_basis(basis.Molecule(["H"], np.zeros((1, 3))),
                            basis.read_basfile(write(tmp_path, "h2.dat", txt.replace("D0", "").replace("d0", ""))))
    same_shells(ns.shells, py)


@pytest.mark.parametrize("case,match", [
    ("missing", "cannot open"),
    ("element", "element not recognized"),
    ("notinbasis", "not in basis"),
    ("header", "unknown header line"),
    ("short", "unexpected end of file"),
])
def test_errors_are_reported(tmp_path, case, match):
    good = "2\ntitle\nUSEDENSITYSUPGUESS Y\nH 0.0 0.0 0.0\nH 0.0 0.0 0.74\n"
    inp = {"missing": str(tmp_path / "nope.inp"),
           "element": write(tmp_path, "a.inp", good.replace("H 0.0 0.0 0.74", "Xx 0.0 0.0 0.74")),
           "notinbasis": write(tmp_path, "b.inp", good.replace("H 0.0 0.0 0.74", "Ar 0.0 0.0 0.74")),
           "header": write(tmp_path, "c.inp", good.replace("USEDENSITYSUPGUESS", "FOO")),
           "short": write(tmp_path, "d.inp", good.replace("H 0.0 0.0 0.74\n", ""))}[case]
    with pytest.raises(HfgpuError, match=match):
        ingest.load_system("STO-3G", infile=inp)


@pytest.mark.gpu
def test_scf_on_native_ingestion_matches_python_ingestion():
    """Water in 6-31G(d), read by the C++ layer from the reference's own
    h2oc.inp, runs through the CUDA builder and the SCF; the energy equals
    the one from the Python-read shells to 1e-10 Eh."""
    from hfcode_b200 import scf
    from hfcode_b200.fock import FockBuilder
    path = os.path.join(INP, "h2oc.inp")
    res = []
    for native in (True, False):
        if native:
            ns = ingest.load_system("6-31G(d)", infile=path)
            mol, sh, p0 = ns.mol, ns.shells, ns.p_guess
        else:
            mol, _, sh, p0 = python_side("6-31G(d)", infile=path)
        fb = FockBuilder(sh)
        r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60)
        fb.close()
        assert r.converged
        res.append(r.energy)
    assert abs(res[0] - res[1]) < 1e-10
