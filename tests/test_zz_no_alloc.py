"""The no-allocation entry point hfgpu_fock_build_diag_static, through the C ABI.

Some callers cannot allocate GPU memory where they call the Fock builder --
code running where cudaMalloc is not permitted, or that must keep the device
footprint fixed after start-up.  hfgpu_fock_build_diag_static serves them: it
runs fock_build_diag on device pointers with its scratch in a static device
array.  This file is collected last so that a failure here comes after every
other test has run; it passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from helpers import perturbed_density, system

TOL = 1e-10  # the FP64 element tolerance of the parity tests


@pytest.mark.gpu
def test_static_scratch_diag_matches_fock_build_diag():
    import torch

    from hfcode_b200 import fock
    from oracle import pyoracle

    _, _, sh, p0 = system("benzene")
    nb = sh.nb
    fb = fock.FockBuilder(sh)
    f0 = np.zeros((nb, nb))
    fb.fock_build_initial_diag(f0, p0, 1e-10)
    orc = pyoracle.Oracle(sh)  # the CPU restatement of fock_build_diag, as a second check
    orc.fock_build_initial_diag(np.zeros((nb, nb)), p0, 1e-10)
    dev = torch.device("cuda", torch.cuda.current_device())
    for call, seed in enumerate((5, 6)):  # two calls in a row share the scratch
        p = perturbed_density(p0, seed)
        ref = np.full((nb, nb), 0.5)
        fb.fock_build_diag(ref, p, 1e-10)
        P = torch.from_numpy(np.ascontiguousarray(p)).to(dev)
        F = torch.full((nb, nb), 0.5, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        fb.fock_build_diag_static(F.data_ptr(), P.data_ptr(), 1e-10)
        ctypes.CDLL(fock.LIBPATH)  # library stays loaded
        torch.cuda.synchronize()
        got = F.cpu().numpy()
        assert np.max(np.abs(got - ref)) < TOL, (call, np.max(np.abs(got - ref)))
        fo = np.full((nb, nb), 0.5)
        orc.fock_build_diag(fo, p, 1e-10)
        assert np.max(np.abs(got - fo)) < TOL, (call, np.max(np.abs(got - fo)))
    fb.close()


@pytest.mark.gpu
def test_static_scratch_rejects_sizes_beyond_its_limit():
    import torch

    from hfcode_b200 import basis, fock, molecules

    mol = molecules.alkane(80)  # nb 1444 > 1024, nsh 644 > 512
    sh = basis.spread_basis(mol, basis.load_basis("6-31G(d)"))
    fb = fock.FockBuilder(sh)
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(fock.HfgpuError, match="exceeds the static scratch limit"):
        fb.fock_build_diag_static(x.data_ptr(), x.data_ptr(), 1e-10)
    fb.close()
