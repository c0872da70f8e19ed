"""The reference's molecule inputs load in every header variant it ships:
the current ten-line header (h2oc, h2ob), a header without DIRECTSCF and with
CRLF line ends (c20h42), and the older HUCKEL headers (benzene, o).  The
files under tests/golden/inputs are copies of the reference's own inputs."""
import os

import numpy as np
import pytest

from hfcode_b200 import basis, inputs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "inputs")


def test_current_header():
    mol, opt = inputs.read_infile(os.path.join(HERE, "h2oc.inp"))
    assert mol.labels == ["O", "H", "H"]
    assert np.allclose(mol.coords_ang[1], [0.71162062, 0.55099555, 0.0])
    assert opt.densup and not opt.directscf and opt.levshft and opt.lshft == 0.4
    assert not opt.uhf and opt.ncore == 1 and opt.prtlevl == 2
    mol_b, opt_b = inputs.read_infile(os.path.join(HERE, "h2ob.inp"))
    assert not opt_b.densup and opt_b.directscf


def test_header_without_directscf_and_crlf():
    mol, opt = inputs.read_infile(os.path.join(HERE, "c20h42.inp"))
    assert len(mol.labels) == 62 and mol.labels.count("C") == 20
    assert "DIRECTSCF" not in opt.keywords and opt.directscf  # default
    assert opt.densup and not opt.levshft and opt.ncore == 5


@pytest.mark.parametrize("name,natom", [("benzene", 12), ("o", 1)])
def test_older_headers(name, natom):
    mol, opt = inputs.read_infile(os.path.join(HERE, f"{name}.inp"))
    assert len(mol.labels) == natom
    assert "HUCKEL" in opt.keywords


def test_loaded_geometry_builds_shells():
    mol, _ = inputs.read_infile(os.path.join(HERE, "benzene.inp"))
    sh = basis.spread_basis(mol, basis.load_basis("6-31G(d)"))
    assert sh.nb == 96 and mol.nocc == 21
