"""Batching form: a full build recorded once as a CUDA graph and replayed.

The replay must give the same F as the separate fock_build_diag +
fock_build_non_diag calls (same kernels and screening; only the order of the
FP64 atomic sums differs, so 1e-11 absolute on F), must read P at replay
time (a second density through the same capture), and a batch of several
molecules' captures in one launch must give each molecule's own F.  The SCF
driver with graph replays must reach the golden energy (1e-8 Eh)."""
import json
import os

import numpy as np
import pytest

from helpers import perturbed_density, system
from hfcode_b200 import scf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FTOL = 1e-11


def eager(fb, p, thr_d, thr_n, cut=0.0):
    f = np.zeros((fb.nb, fb.nb))
    fb.fock_build_diag(f, p, thr_d)
    if cut > 0.0:
        fb.fock_build_non_diag_mixed(f, p, thr_n, cut)
    else:
        fb.fock_build_non_diag(f, p, thr_n)
    return f


def ready(name):
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system(name)
    fb = FockBuilder(sh)
    fb.fock_build_initial_diag(np.zeros((sh.nb, sh.nb)), p0, 1e-10)
    return fb, p0


@pytest.mark.gpu
@pytest.mark.parametrize("cut", [0.0, 1e-6])
def test_graph_replay_matches_separate_calls(cut):
    fb, p0 = ready("benzene")
    for seed in (1, 2):  # the second density goes through the same capture
        p = perturbed_density(p0, seed)
        ref = eager(fb, p, 1e-10, 1e-11, cut)
        f = np.zeros_like(ref)
        fb.fock_build_graph(f, p, 1e-10, 1e-11, cut)
        assert np.max(np.abs(f - ref)) < FTOL
        if cut > 0.0:
            assert fb.class_stats()["fp32"].sum() > 0
    fb.close()


@pytest.mark.gpu
def test_graph_accumulates_into_f():
    fb, p0 = ready("alkane2")
    h = np.random.default_rng(3).normal(size=(fb.nb, fb.nb))
    h = h + h.T
    ref = h + eager(fb, p0, 1e-10, 1e-10)
    f = h.copy()
    fb.fock_build_graph(f, p0, 1e-10, 1e-10)
    assert np.max(np.abs(f - ref)) < FTOL
    fb.close()


@pytest.mark.gpu
def test_batch_of_captures_matches_each_molecule():
    import torch
    from hfcode_b200.fock import Batch
    names = ["alkane1", "water", "benzene", "alkane3"]
    fbs, refs, bufs = [], [], []
    for i, name in enumerate(names):
        fb, p0 = ready(name)
        p = perturbed_density(p0, 10 + i)
        refs.append(eager(fb, p, 1e-10, 1e-10))
        P = torch.tensor(np.asfortranarray(p).ravel(order="F"), dtype=torch.float64, device="cuda")
        F = torch.zeros(fb.nb * fb.nb, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        fb.graph_capture(F.data_ptr(), P.data_ptr(), 1e-10, 1e-10)
        fbs.append(fb)
        bufs.append((F, P))
    batch = Batch(fbs)
    for rep in range(2):  # F accumulates: zero it before each replay
        for F, _ in bufs:
            F.zero_()
        torch.cuda.synchronize()
        batch.launch(0)
        torch.cuda.synchronize()
        for fb, ref, (F, _) in zip(fbs, refs, bufs):
            f = F.cpu().numpy().reshape(fb.nb, fb.nb, order="F")
            assert np.max(np.abs(f - ref)) < FTOL
    batch.close()
    for fb in fbs:
        fb.close()


@pytest.mark.gpu
def test_single_capture_launch_on_device_pointers():
    import torch
    fb, p0 = ready("alkane2")
    p = perturbed_density(p0, 5)
    ref = eager(fb, p, 1e-10, 1e-10, 1e-7)
    P = torch.tensor(np.asfortranarray(p).ravel(order="F"), dtype=torch.float64, device="cuda")
    F = torch.zeros(fb.nb * fb.nb, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fb.graph_capture(F.data_ptr(), P.data_ptr(), 1e-10, 1e-10, 1e-7)
    fb.graph_launch()
    fb.synchronize()
    f = F.cpu().numpy().reshape(fb.nb, fb.nb, order="F")
    assert np.max(np.abs(f - ref)) < 1e-10
    fb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "benzene"])
def test_scf_with_graph_replays_matches_golden(name):
    from hfcode_b200.fock import FockBuilder
    gold = json.load(open(os.path.join(GOLD, "energies.json")))[name]
    mol, _, sh, p0 = system(name)
    fb = FockBuilder(sh)
    r = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-10, conv=1e-7, maxiter=60, graph=True)
    fb.close()
    assert r.converged
    assert abs(r.energy - gold["energy"]) < 1e-8, (r.energy, gold["energy"])
