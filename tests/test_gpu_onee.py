"""One-electron integrals on the GPU (hfgpu_one_electron_gpu) against the
host restatement (hfgpu_one_electron, itself checked in test_oracle.py):
S, T, V element-wise for s, p, l and d shells, up to C60."""
import numpy as np
import pytest

from helpers import system
from hfcode_b200 import basis, molecules, onee


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "benzene", "benzene_sp", "alkane2_mix", "c60"])
def test_gpu_one_electron_matches_host(name):
    if name == "c60":
        mol = molecules.c60()
        sh = basis.spread_basis(mol, basis.load_basis("6-31G(d)"))
    else:
        mol, _, sh, _ = system(name)
    host = onee.one_electron(mol, sh)
    dev = onee.one_electron(mol, sh, gpu=True)
    for h, d in zip(host, dev):
        scale = max(1.0, np.max(np.abs(h)))
        assert np.max(np.abs(h - d)) < 1e-12 * scale
