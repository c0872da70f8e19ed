"""Reads the reference's molecule input files (`*.inp`).

read_infile.f90:12-61 expects ten header lines -- natom, title,
USEDENSITYSUPGUESS, DIRECTSCF, LEVELSHIFT (flag, shift), UHF (flag, 2S),
MP2, CCSD, PRINT, ncore -- and then one line per atom (label, x, y, z in
Angstrom).  Most inputs the reference ships use older headers: HUCKEL in
place of the density-guess and direct flags, or no DIRECTSCF line, and some
have CRLF line ends.  This reader takes the keyword lines in any order until
the first atom line, so every variant loads; options missing from a file
get the defaults below.
"""
from __future__ import annotations

import dataclasses
from typing import List

import numpy as np

from .basis import Molecule


@dataclasses.dataclass
class InputOptions:
    title: str = ""
    densup: bool = False        # USEDENSITYSUPGUESS: atomic-density guess
    directscf: bool = True      # DIRECTSCF
    levshft: bool = False       # LEVELSHIFT flag
    lshft: float = 0.0          # LEVELSHIFT value
    uhf: bool = False
    sz: int = 0
    mp2: bool = False
    ccsd: bool = False
    huckel: bool = False        # older files: HUCKEL guess flag
    prtlevl: int = 0
    ncore: int = 0
    keywords: List[str] = dataclasses.field(default_factory=list)  # header keywords as found


def _yes(tok: str) -> bool:
    return tok.strip().lower().startswith("y")


def _is_atom_line(toks) -> bool:
    if len(toks) < 4:
        return False
    try:
        [float(t) for t in toks[1:4]]
    except ValueError:
        return False
    return toks[0][0].isalpha()


def read_infile(path: str):
    """(Molecule, InputOptions) from a reference input file, any header variant."""
    with open(path, "r", newline=None) as fh:
        lines = [ln.strip() for ln in fh.read().splitlines()]
    lines = [ln for ln in lines if ln]
    natom = int(lines[0].split()[0])
    opt = InputOptions(title=lines[1])
    i = 2
    while i < len(lines) and not _is_atom_line(lines[i].split()):
        toks = lines[i].split()
        key = toks[0].upper()
        opt.keywords.append(key)
        arg = toks[1:] + ["", ""]
        if key == "USEDENSITYSUPGUESS":
            opt.densup = _yes(arg[0])
        elif key == "DIRECTSCF":
            opt.directscf = _yes(arg[0])
        elif key == "LEVELSHIFT":
            opt.levshft = _yes(arg[0])
            opt.lshft = float(arg[1]) if arg[1] else 0.0
        elif key == "UHF":
            opt.uhf = _yes(arg[0])
            opt.sz = int(arg[1]) if arg[1] else 0
        elif key == "MP2":
            opt.mp2 = _yes(arg[0])
        elif key == "CCSD":
            opt.ccsd = _yes(arg[0])
        elif key == "HUCKEL":
            opt.huckel = _yes(arg[0])
        elif key == "PRINT":
            opt.prtlevl = int(arg[0])
        elif key == "NCORE":
            opt.ncore = int(arg[0])
        else:
            raise ValueError(f"{path}: unknown header line {lines[i]!r}")
        i += 1
    labels, xyz = [], []
    for ln in lines[i:i + natom]:
        toks = ln.split()
        if not _is_atom_line(toks):
            raise ValueError(f"{path}: bad atom line {ln!r}")
        labels.append(toks[0].capitalize())
        xyz.append([float(t) for t in toks[1:4]])
    if len(labels) != natom:
        raise ValueError(f"{path}: {natom} atoms announced, {len(labels)} found")
    return Molecule(labels, np.array(xyz)), opt
