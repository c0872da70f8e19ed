"""CUDA Fock builds against the CPU oracle, through the C ABI.

Tolerance: 1e-10 absolute on every Fock element (the FP64 contract), on the
same inputs.  Both sides apply the reference's screening, so the per-class
counts of screened-in quartets must agree as well.
"""
import numpy as np
import pytest

from helpers import perturbed_density, system
from oracle import pyoracle

TOL = 1e-10
# reference pair classes (ss sp sd sl pp pd pl dd dl ll) -> GPU pair types
# (SS LS LL DS DL DD PS LP PP DP)
REF2GPU = {0: 0, 3: 1, 9: 2, 2: 3, 8: 4, 7: 5, 1: 6, 6: 7, 4: 8, 5: 9}


def gpu_class(ti, tj):
    from hfcode_b200.fock import CLASS_NAMES, PAIR_TYPES
    a, b = min(ti, tj), max(ti, tj)
    return CLASS_NAMES.index(f"{PAIR_TYPES[a]}|{PAIR_TYPES[b]}")


def oracle_counts_by_gpu_class(orc):
    passed, _ = orc.counts()
    from hfcode_b200.fock import NCLASS
    out = np.zeros(NCLASS, dtype=np.int64)
    for ca in range(10):
        for cb in range(10):
            if passed[ca, cb]:
                out[gpu_class(REF2GPU[ca], REF2GPU[cb])] += passed[ca, cb]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water", "alkane1", "alkane2", "benzene", "water_sp", "alkane2_sp", "alkane2_mix",
                                  "h2", "ne"])
def test_fock_build_parity(name):
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system(name)
    nb = sh.nb
    fb = FockBuilder(sh)
    orc = pyoracle.Oracle(sh)
    h = np.random.default_rng(1).normal(size=(nb, nb))
    h = h + h.T
    thr = 1e-10
    # cycle 1: initial diag + non-diag
    fg, fo = h.copy(order="F"), h.copy(order="F")
    fb.fock_build_initial_diag(fg, p0, thr)
    orc.fock_build_initial_diag(fo, p0, thr)
    assert np.max(np.abs(fg - fo)) < TOL
    sg, lastg = fb.schwarz()
    so, lasto = orc.schwarz()
    assert lastg == lasto
    assert np.max(np.abs(sg - so)) < 1e-12
    fb.fock_build_non_diag(fg, p0, thr)
    orc.fock_build_non_diag(fo, p0, thr)
    assert np.max(np.abs(fg - fo)) < TOL
    st = fb.class_stats()
    assert np.array_equal(st["pass"], oracle_counts_by_gpu_class(orc))
    # later cycle: diag + non-diag on another density, and the incremental
    # (delta-P, thr/10) build of direct_hartreefock.f90:111-121
    p1 = perturbed_density(p0, 2)
    fg, fo = h.copy(order="F"), h.copy(order="F")
    fb.fock_build_diag(fg, p1, thr)
    orc.fock_build_diag(fo, p1, thr)
    assert np.max(np.abs(fg - fo)) < TOL
    fb.fock_build_non_diag(fg, p1, thr)
    orc.fock_build_non_diag(fo, p1, thr)
    assert np.max(np.abs(fg - fo)) < TOL
    dp = p1 - p0
    dg, do = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_diag(dg, dp, thr)
    orc.fock_build_diag(do, dp, thr)
    fb.fock_build_non_diag(dg, dp, thr * 0.1)
    orc.fock_build_non_diag(do, dp, thr * 0.1)
    assert np.max(np.abs(dg - do)) < TOL
    # J only
    jg, jo = np.zeros((nb, nb)), np.zeros((nb, nb))
    fb.fock_build_non_diag_j_only(jg, p1, thr)
    orc.fock_build_non_diag_j_only(jo, p1, thr)
    assert np.max(np.abs(jg - jo)) < TOL
    fb.close()


@pytest.mark.gpu
def test_fock_build_is_symmetric_and_accumulates():
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system("benzene")
    fb = FockBuilder(sh)
    nb = sh.nb
    f1 = np.zeros((nb, nb))
    fb.fock_build_initial_diag(f1, p0, 1e-10)
    fb.fock_build_non_diag(f1, p0, 1e-10)
    assert np.max(np.abs(f1 - f1.T)) < 1e-13
    f2 = np.full((nb, nb), 3.0)
    fb.fock_build_diag(f2, p0, 1e-10)
    fb.fock_build_non_diag(f2, p0, 1e-10)
    f3 = np.zeros((nb, nb))
    fb.fock_build_diag(f3, p0, 1e-10)
    fb.fock_build_non_diag(f3, p0, 1e-10)
    assert np.max(np.abs(f2 - 3.0 - f3)) < 1e-12
    fb.close()


@pytest.mark.gpu
def test_calls_before_initial_diag_are_rejected():
    from hfcode_b200.fock import FockBuilder, HfgpuError
    _, _, sh, p0 = system("water")
    fb = FockBuilder(sh)
    with pytest.raises(HfgpuError):
        fb.fock_build_non_diag(np.zeros((sh.nb, sh.nb)), p0, 1e-10)
    fb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["zero_density", "one_atom_block", "thr_zero", "thr_huge"])
def test_edge_densities_and_thresholds(case):
    """Ragged and degenerate inputs: P = 0 and a threshold above every bound
    (every quartet screened out: empty class lists, F left exactly as it
    was), a density with one atom's block only (most shell pairs screened
    out, a few classes active), and thr = 0 (nothing dropped by either
    screen).  Parity and the per-class counts against the oracle."""
    from hfcode_b200.fock import FockBuilder
    name = "alkane1" if case == "thr_zero" else "benzene"
    _, _, sh, p0 = system(name)
    nb = sh.nb
    fb = FockBuilder(sh)
    orc = pyoracle.Oracle(sh)
    fb.fock_build_initial_diag(np.zeros((nb, nb)), p0, 1e-10)
    orc.fock_build_initial_diag(np.zeros((nb, nb)), p0, 1e-10)
    thr = {"thr_zero": 0.0, "thr_huge": 1e3}.get(case, 1e-10)
    if case == "zero_density":
        p = np.zeros((nb, nb))
    elif case == "one_atom_block":
        n0 = int(sh.nbfsat[0])
        p = np.zeros((nb, nb))
        p[:n0, :n0] = perturbed_density(p0, 4)[:n0, :n0]
    else:
        p = perturbed_density(p0, 4)
    h = np.random.default_rng(5).normal(size=(nb, nb))
    h = h + h.T
    fg, fo = h.copy(order="F"), h.copy(order="F")
    for f, b in ((fg, fb), (fo, orc)):
        b.fock_build_diag(f, p, thr)
        b.fock_build_non_diag(f, p, thr)
    st = fb.class_stats()
    assert np.array_equal(st["pass"], oracle_counts_by_gpu_class(orc))
    if case in ("zero_density", "thr_huge"):
        assert st["pass"].sum() == 0
        assert np.array_equal(fg, h)
    else:
        assert st["pass"].sum() > 0
        assert np.max(np.abs(fg - fo)) < TOL
    fb.close()


@pytest.mark.gpu
def test_default_scratch_follows_the_molecule():
    """The default scratch budget (24 GiB) is an upper bound: a handle
    allocates only what its largest class list needs, so a small molecule's
    device footprint stays small, and a tight explicit budget (more chunks)
    gives the same F."""
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system("benzene")
    nb = sh.nb
    out = []
    for budget in (None, 1 << 20):
        fb = FockBuilder(sh, scratch_budget=budget)
        f = np.zeros((nb, nb))
        fb.fock_build_initial_diag(f, p0, 1e-10)
        fb.fock_build_non_diag(f, p0, 1e-10)
        if budget is None:
            assert fb.device_bytes() < (256 << 20)
        out.append(f)
        fb.close()
    assert np.max(np.abs(out[0] - out[1])) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["benzene", "alkane2_mix"])
def test_merged_and_separate_role_launches_agree(name):
    """Small chunks run every role of a stage in one launch (gridDim.y =
    roles); HFGPU_MERGE_BLOCKS=0 at handle creation forces one launch per
    role.  Both give the oracle's F and agree with each other to rounding."""
    import os
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system(name)
    nb = sh.nb
    p = perturbed_density(p0, 9)
    out = {}
    old = os.environ.get("HFGPU_MERGE_BLOCKS")
    try:
        for label, val in (("separate", "0"), ("merged", "1000000")):
            os.environ["HFGPU_MERGE_BLOCKS"] = val
            fb = FockBuilder(sh)
            f = np.zeros((nb, nb))
            fb.fock_build_initial_diag(f, p0, 1e-10)
            fb.fock_build_non_diag(f, p, 1e-10)
            fb.fock_build_non_diag_mixed(f, p, 1e-10, 1e-6)
            out[label] = (f, fb.launch_count())
            fb.close()
    finally:
        if old is None:
            os.environ.pop("HFGPU_MERGE_BLOCKS", None)
        else:
            os.environ["HFGPU_MERGE_BLOCKS"] = old
    assert np.max(np.abs(out["separate"][0] - out["merged"][0])) < 1e-11
    assert out["merged"][1] < out["separate"][1]  # fewer launches


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["benzene", "alkane2_mix"])
def test_grouped_and_single_thread_scatter_agree(name):
    """The staged scatter runs one thread per quartet, or four lanes per
    quartet where the class's tuning chooses it; HFGPU_SCATTER at handle
    creation forces one form everywhere.  FP64 builds and mixed builds (FP32
    chunks below the cutoff) of both forms agree to rounding, and the FP64
    builds match the oracle."""
    import os
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system(name)
    nb = sh.nb
    p = perturbed_density(p0, 10)
    out = {}
    old = os.environ.get("HFGPU_SCATTER")
    try:
        for mode in ("single", "grouped"):
            os.environ["HFGPU_SCATTER"] = mode
            fb = FockBuilder(sh)
            f64 = np.zeros((nb, nb))
            fb.fock_build_initial_diag(f64, p0, 1e-10)
            fb.fock_build_non_diag(f64, p, 1e-10)
            fmx = np.zeros((nb, nb))
            fb.fock_build_non_diag_mixed(fmx, p, 1e-10, 1e3)  # every quartet in FP32
            out[mode] = (f64, fmx)
            fb.close()
    finally:
        if old is None:
            os.environ.pop("HFGPU_SCATTER", None)
        else:
            os.environ["HFGPU_SCATTER"] = old
    orc = pyoracle.Oracle(sh)
    fo = np.zeros((nb, nb), order="F")
    orc.fock_build_initial_diag(fo, p0, 1e-10)
    orc.fock_build_non_diag(fo, p, 1e-10)
    assert np.max(np.abs(out["single"][0] - out["grouped"][0])) < 1e-12
    assert np.max(np.abs(out["grouped"][0] - fo)) < 1e-10
    # FP32 block sums: the two forms add the same FP32 products in different orders
    scale = max(1.0, float(np.max(np.abs(out["single"][1]))))
    assert np.max(np.abs(out["single"][1] - out["grouped"][1])) < 1e-5 * scale


@pytest.mark.gpu
def test_class_stream_count_does_not_change_f():
    """HFGPU_STREAMS (read at handle creation) spreads the classes over one to
    eight concurrent streams, each with its own scratch slot.  The F of one
    and of eight streams agree to rounding and match the oracle."""
    import os
    from hfcode_b200.fock import FockBuilder
    _, _, sh, p0 = system("alkane2_mix")
    nb = sh.nb
    p = perturbed_density(p0, 11)
    out = {}
    old = os.environ.get("HFGPU_STREAMS")
    try:
        for n in ("1", "8"):
            os.environ["HFGPU_STREAMS"] = n
            fb = FockBuilder(sh)
            f = np.zeros((nb, nb))
            fb.fock_build_initial_diag(f, p0, 1e-10)
            fb.fock_build_non_diag(f, p, 1e-10)
            out[n] = f
            fb.close()
    finally:
        if old is None:
            os.environ.pop("HFGPU_STREAMS", None)
        else:
            os.environ["HFGPU_STREAMS"] = old
    orc = pyoracle.Oracle(sh)
    fo = np.zeros((nb, nb), order="F")
    orc.fock_build_initial_diag(fo, p0, 1e-10)
    orc.fock_build_non_diag(fo, p, 1e-10)
    assert np.max(np.abs(out["1"] - out["8"])) < 1e-12
    assert np.max(np.abs(out["8"] - fo)) < 1e-10
