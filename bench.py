"""Benchmark: Fock builds/s for C60/6-31G(d) on one B200.

One step = one full Fock build at a fixed density: fock_build_diag +
fock_build_non_diag at thr = 1e-10 (the reference's definition of a build,
direct_hartreefock.f90:106-110), excluding the once-per-SCF set-up
(hfgpu_init + fock_build_initial_diag).

  value   device-resident builds/s (F, P in HBM; hfgpu_fock_build_device)
  e2e     the same build through the reference-facing C ABI with HOST
          buffers (fock_build_diag + fock_build_non_diag, H2D/D2H included)
  roofline  the dominant quartet-class kernel against the measured FP64 FMA
          peak of the device
  cpu_baseline  the CPU oracle (a restatement of the reference's Fortran) on
          the host cores, on a bounded row sample of the same build

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Under torchrun each rank runs an independent replica on its own GPU (the
builder is single-GPU by design); value is the sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Fock builds/s, C60/6-31G(d)"
THR = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--molecule", default="c60")
    ap.add_argument("--density", default="core_guess", choices=["core_guess", "atomic_guess"],
                    help="core-Hamiltonian guess (dense, direct_hartreefock.f90:61-91) or the atomic-density "
                         "guess (block-diagonal, :50-59)")
    ap.add_argument("--cpu-stride", type=int, default=16,
                    help="CPU legs: each step builds the bra rows ii %% stride == 0 of every class block")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP64-vs-mixed SCF study")
    ap.add_argument("--mixed-cutoffs", default="1e-7,1e-5,1e-3")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream study")
    ap.add_argument("--serve-jobs", type=int, default=1000)
    ap.add_argument("--serve-rate", type=float, default=12.0, help="Poisson arrival rate of the served stream")
    ap.add_argument("--serve-plain", type=int, default=100, help="jobs of the one-at-a-time comparison")
    ap.add_argument("--cutoff", type=float, default=0.0,
                    help="FP32 cutoff of the timed build (0 = the FP64 build the metric is quoted on)")
    return ap.parse_args()


def workload(name: str, density: str, oracle_side: bool = False):
    """Molecule, shells and the fixed density of one bench step.  The core
    guess needs S, T, V: the GPU arm takes them from this library, the CPU
    reference arm from the oracle (oracle/oscf.py), so that arm never loads
    libhfgpu.so; both give the same density to rounding."""
    from hfcode_b200 import basis, molecules
    if name == "c60":
        mol, bas = molecules.c60(), basis.load_basis("6-31G(d)")
        label = "C60/6-31G(d)"
    elif name == "benzene":
        mol, bas = molecules.benzene(), basis.load_basis("6-31G(d)")
        label = "benzene/6-31G(d)"
    else:
        n = int(name[1:name.index("h")])
        mol, bas = molecules.alkane(n), basis.load_basis("6-31G(d)")
        label = f"C{n}H{2 * n + 2}/6-31G(d)"
    sh = basis.spread_basis(mol, bas)
    if density == "atomic_guess":
        p = basis.density_superposition(mol, bas, sh.nb)
    elif oracle_side:
        from oracle import oscf
        p = oscf.OracleSCF(mol.charges, mol.coords, mol.nocc, sh).core_density()
    else:
        from hfcode_b200 import onee
        p = onee.core_density(mol, sh)
    return label, mol, sh, p


def bench_config(label: str, nb: int, density: str, world: int) -> dict:
    """The workload description, identical in the GPU arm and the reference arm."""
    return {"workload": f"{label} one Fock build (fock_build_diag + fock_build_non_diag), thr=1e-10",
            "nb": nb, "density": density, "parallelism": f"replicas{world}",
            "l2": "GPU arm: flushed between steps (256 MiB write outside the timed events)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_builds(sh, p, warmup: int, steps: int, stride: int, calibrate: bool = True) -> dict:
    """The oracle (a C++/OpenMP restatement of the reference's builders) on
    all host cores.  Each step is fock_build_diag in full plus
    fock_build_non_diag on the same fixed rows every step: the bra rows
    ii % stride == 0 of every class block (the rows are in descending Schwarz
    order, so this is a stratified 1/stride sample).  One unsampled
    fock_build_non_diag, timed once after the steps, calibrates the
    extrapolation: ratio = t_full / (stride * t_sample)."""
    from oracle import pyoracle
    orc = pyoracle.Oracle(sh)
    nb = sh.nb
    f = np.zeros((nb, nb))
    orc.fock_build_initial_diag(f, p, THR)
    td, ts = [], []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        orc.fock_build_diag(f, p, THR)
        t1 = time.perf_counter()
        n = orc.fock_build_non_diag_sample(f, p, THR, stride, 0)
        t2 = time.perf_counter()
        if it >= warmup:
            td.append(t1 - t0)
            ts.append(t2 - t1)
    t_diag, t_samp = float(np.median(td)), float(np.median(ts))
    cal = {"ratio": 1.0, "full_non_diag_s": None}
    if calibrate:
        t0 = time.perf_counter()
        orc.fock_build_non_diag(f, p, THR)
        t_full = time.perf_counter() - t0
        cal = {"ratio": t_full / (stride * t_samp), "full_non_diag_s": t_full,
               "sampled_non_diag_s": t_samp, "stride": stride}
    t_build = t_diag + stride * t_samp * cal["ratio"]
    threads = pyoracle.lib().orc_num_threads()
    return {"value": 1.0 / t_build, "unit": "builds/s", "cores": threads, "kind": "port", "extrapolated": True,
            "step_seconds": t_diag + t_samp, "calibration": cal,
            "sample": f"each step: fock_build_diag in full + fock_build_non_diag on the fixed bra rows ii % {stride} "
                      f"== 0 of every class block ({n} screened-in quartets); extrapolated x{stride} times the "
                      f"calibration ratio of one unsampled build in the same run"}


def mixed_study(fock, mol, sh, cutoffs, dev):
    """FP64 vs mixed precision on the SCF path.

    * converged energies of the reference protocol (conve 1e-9) with FP64 and
      with mixed incremental builds, |dE| against the FP64 run and against
      the oracle's FP64 energy (golden fixture);
    * the speed of one incremental (delta-P) build near convergence in both
      forms, with max|dF| between them;
    * the whole SCF with the job's state on the device (the library's C++
      step), FP64 and mixed alternating three times each;
    * one full build at the converged density;
    * n-C20H42 (the configuration the mixed target is quoted on) at cutoff
      1e-7: its incremental-build speed-up and |dE| against the oracle."""
    import torch
    from hfcode_b200 import basis, onee, scf
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "energies.json")))
    bas = basis.load_basis("6-31G(d)")
    p0 = basis.density_superposition(mol, bas, sh.nb)
    ints = onee.one_electron(mol, sh, gpu=True)
    out = {"cutoffs": {}}
    fb = fock.FockBuilder(sh)
    t0 = time.perf_counter()
    r64 = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80, ints=ints)
    out["scf_fp64"] = {"energy": r64.energy, "cycles": r64.cycles, "converged": r64.converged,
                       "seconds": time.perf_counter() - t0,
                       "abs_dE_vs_oracle": abs(r64.energy - gold["c60"]["energy"]) if sh.nb == 840 else None}
    # the whole SCF on the device (C++ step), after one small warm-up SCF so
    # that neither form carries the libraries' first-call costs
    from hfcode_b200 import molecules
    wmol = molecules.benzene()
    wsh = basis.spread_basis(wmol, bas)
    fbw = fock.FockBuilder(wsh)
    scf.device_hartreefock(wmol, wsh, fbw, p_guess=basis.density_superposition(wmol, bas, wsh.nb), conve=1e-9,
                           conv=1e-6, maxiter=80, fp32_cutoff=1e-5)
    fbw.close()
    # and one untimed SCF of this molecule: the stream-ordered memory pool
    # grows to this job's size once, instead of inside the first timed run
    fbw = fock.FockBuilder(sh)
    scf.device_hartreefock(mol, sh, fbw, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80, ints=ints)
    fbw.close()
    for rep in range(3):
        for label, cut in (("device_scf_fp64", 0.0), ("device_scf_mixed_1e-05", 1e-5)):
            fbd = fock.FockBuilder(sh)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            rd = scf.device_hartreefock(mol, sh, fbd, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80,
                                        fp32_cutoff=cut, ints=ints)
            sec = time.perf_counter() - t1
            fbd.close()
            runs = out.get(label, {}).get("runs_seconds", []) + [sec]
            out[label] = {"energy": rd.energy, "cycles": rd.cycles, "converged": rd.converged,
                          "seconds": float(np.median(runs)), "runs_seconds": runs,
                          "spread": (max(runs) - min(runs)) / min(runs),
                          "abs_dE_vs_host_fp64": abs(rd.energy - r64.energy),
                          "scf_builds_per_s": rd.cycles / float(np.median(runs))}
    nb = sh.nb
    stream = torch.cuda.ExternalStream(fb.stream(), device=dev)
    F = torch.zeros((nb, nb), dtype=torch.float64, device=dev)

    def timed(P, thr_nd, cut, reps=3):
        ts = []
        for _ in range(reps + 1):
            F.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fb.fock_build_device(F.data_ptr(), P.data_ptr(), THR, thr_nd, cut)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts[1:])), F.cpu().numpy().copy(), fb.class_stats()

    # a full build at the converged density
    Pc = torch.from_numpy(np.ascontiguousarray(r64.P)).to(dev)
    tc, _, stc = timed(Pc, THR, 0.0)
    out["converged_density_build"] = {"ms": tc, "builds_per_s": 1000.0 / tc,
                                      "screened_in_quartets": int(stc["pass"].sum())}
    # a delta-P near convergence: the one-cycle update of the converged density
    X = onee.s_minus_half(ints[0])
    _, C = np.linalg.eigh(X @ r64.F @ X.T)
    C = X @ C
    p_next = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T
    dp = p_next - r64.P
    out["delta_p_max"] = float(np.max(np.abs(dp)))
    P = torch.from_numpy(np.ascontiguousarray(dp)).to(dev)
    t64, f64, _ = timed(P, THR * 0.1, 0.0)
    out["delta_build_ms_fp64"] = t64
    for cut in cutoffs:
        tm, fm, stm = timed(P, THR * 0.1, cut)
        fbm = fock.FockBuilder(sh)
        t1 = time.perf_counter()
        rm = scf.direct_hartreefock(mol, sh, fbm, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80, ints=ints,
                                    fp32_cutoff=cut)
        fbm.close()
        out["cutoffs"][f"{cut:g}"] = {
            "delta_build_ms": tm, "speedup_vs_fp64": t64 / tm,
            "fp32_quartet_fraction": float(stm["fp32"].sum() / max(1, stm["scattered"].sum())),
            "max_abs_dF_vs_fp64": float(np.max(np.abs(fm - f64))),
            "scf_energy": rm.energy, "abs_dE_vs_fp64": abs(rm.energy - r64.energy), "scf_cycles": rm.cycles,
            "converged": rm.converged, "scf_seconds": time.perf_counter() - t1}
    fb.close()
    out["c20h42_cutoff_1e-07"] = mixed_c20h42(fock, gold["c20h42"], dev)
    return out


def mixed_c20h42(fock, gold, dev):
    """n-C20H42/6-31G(d) with FP32 below bound 1e-7 in the incremental builds:
    delta-P build speed-up against FP64 and the converged SCF energy against
    the oracle's FP64 energy."""
    import torch
    from hfcode_b200 import basis, molecules, onee, scf
    mol = molecules.alkane(20)
    bas = basis.load_basis("6-31G(d)")
    sh = basis.spread_basis(mol, bas)
    p0 = basis.density_superposition(mol, bas, sh.nb)
    ints = onee.one_electron(mol, sh, gpu=True)
    fb = fock.FockBuilder(sh)
    r64 = scf.direct_hartreefock(mol, sh, fb, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80, ints=ints)
    fbm = fock.FockBuilder(sh)
    rm = scf.direct_hartreefock(mol, sh, fbm, p_guess=p0, conve=1e-9, conv=1e-6, maxiter=80, ints=ints,
                                fp32_cutoff=1e-7)
    fbm.close()
    X = onee.s_minus_half(ints[0])
    _, C = np.linalg.eigh(X @ r64.F @ X.T)
    C = X @ C
    dp = 2.0 * C[:, :mol.nocc] @ C[:, :mol.nocc].T - r64.P
    nb = sh.nb
    P = torch.from_numpy(np.ascontiguousarray(dp)).to(dev)
    F = torch.zeros((nb, nb), dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(fb.stream(), device=dev)

    def timed(cut, reps=5):
        ts = []
        for _ in range(reps + 1):
            F.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fb.fock_build_device(F.data_ptr(), P.data_ptr(), THR, THR * 0.1, cut)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts[1:])), F.cpu().numpy().copy()

    t64, f64 = timed(0.0)
    tm, fm = timed(1e-7)
    fb.close()
    return {"nb": nb, "delta_build_ms_fp64": t64, "delta_build_ms_mixed": tm, "speedup_vs_fp64": t64 / tm,
            "max_abs_dF_vs_fp64": float(np.max(np.abs(fm - f64))),
            "scf_energy_fp64": r64.energy, "scf_energy_mixed": rm.energy,
            "abs_dE_mixed_vs_oracle": abs(rm.energy - gold["energy"]),
            "abs_dE_fp64_vs_oracle": abs(r64.energy - gold["energy"])}


def batch_study(fock, dev, reps: int = 5):
    """Batching form on eight served-size molecules (C4H10 ... (H2O)12,
    6-31G(d), atomic-density guess): the wall time of one full build of each,
    (a) one after another through the device entry point (each build enqueues
    its ~100-300 kernels and reads its survivor counts back once), (b) as
    eight CUDA-graph replays, and (c) as one graph launch holding all eight
    instances (hfgpu_batch_launch), with the kernels each launch runs."""
    import torch
    from hfcode_b200 import basis, molecules
    bas = basis.load_basis("6-31G(d)")
    mols = [molecules.alkane(4), molecules.alkane(8), molecules.alkane(12), molecules.alkane(16)] + \
        [molecules.water_cluster(k, np.random.default_rng(k)) for k in (3, 6, 9, 12)]
    fbs, Fs, Ps = [], [], []
    for m in mols:
        sh = basis.spread_basis(m, bas)
        p = basis.density_superposition(m, bas, sh.nb)
        fb = fock.FockBuilder(sh)
        fb.fock_build_initial_diag(np.zeros((sh.nb, sh.nb)), p, THR)
        fbs.append(fb)
        Ps.append(torch.from_numpy(np.ascontiguousarray(p)).to(dev))
        Fs.append(torch.zeros((sh.nb, sh.nb), dtype=torch.float64, device=dev))

    def wall(fn):
        ts = []
        for _ in range(reps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return 1e3 * float(np.median(ts[1:]))

    def eager():
        for fb, F, P in zip(fbs, Fs, Ps):
            fb.fock_build_device(F.data_ptr(), P.data_ptr(), THR, THR, 0.0)

    l0 = sum(fb.launch_count() for fb in fbs)
    t_eager = wall(eager)
    k_eager = (sum(fb.launch_count() for fb in fbs) - l0) / (reps + 1)
    for fb, F, P in zip(fbs, Fs, Ps):
        fb.graph_capture(F.data_ptr(), P.data_ptr(), THR, THR, 0.0)

    def replays():
        for fb in fbs:
            fb.graph_launch()

    t_graph = wall(replays)
    batch = fock.Batch(fbs)
    t_batch = wall(lambda: batch.launch(0))
    batch.close()
    for fb in fbs:
        fb.close()
    return {"molecules": ["C4H10", "C8H18", "C12H26", "C16H34", "(H2O)3", "(H2O)6", "(H2O)9", "(H2O)12"],
            "eager_ms": t_eager, "graph_replays_ms": t_graph, "one_batch_launch_ms": t_batch,
            "kernels_per_round": k_eager, "host_launch_calls": {"eager": k_eager, "graph_replays": len(fbs),
                                                                 "one_batch_launch": 1}}


def served_study(n_jobs: int, rate: float, slots: int, n_plain: int):
    """The serving form: a seeded Poisson stream of RHF/6-31G(d) jobs
    (CnH2n+2 n <= 16, (H2O)k k <= 20; mixed precision at cutoff 1e-7) served
    with continuous batching, every job's state on the device; and the plain
    per-job GPU form (one job at a time, same protocol) on the first
    `n_plain` jobs of the same stream arriving at once."""
    from hfcode_b200 import serve
    jobs = serve.make_stream(n_jobs, rate)
    srv = serve.Server(64 << 30, slots, fp32_cutoff=1e-7)
    srv.warmup()  # one tiny job per slot first (handles, memory pool), outside the stream
    served = srv.serve(jobs)
    plain_jobs = serve.make_stream(n_plain, 0.0)
    plain = serve.serve_sequential(plain_jobs, serve.Server(64 << 30, 1, fp32_cutoff=1e-7))
    sat_jobs = serve.make_stream(n_plain, 0.0)
    sat = serve.Server(64 << 30, slots, fp32_cutoff=1e-7).serve(sat_jobs, realtime=False)
    pick = ("jobs", "jobs_per_s", "makespan_s", "latency_ms")
    return {"stream": {"jobs": n_jobs, "poisson_rate_per_s": rate, "slots": slots, "seed": 20261203,
                       "fp32_cutoff": 1e-7, "state": "device (hfgpu_scf)"},
            "served": {k: served[k] for k in pick + ("service_ms", "queue_ms", "failed", "not_converged",
                                                      "peak_active", "peak_hbm_bytes")},
            "plain_per_job": {k: plain[k] for k in pick},
            "served_all_at_once": {k: sat[k] for k in pick + ("failed",)}}


def run_reference(args):
    """The reference arm: the oracle on the host cores for the same workload,
    density and metric.  It loads only oracle/liboracle.so (the density comes
    from the oracle's own one-electron integrals)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    label, mol, sh, p = workload(args.molecule, args.density, oracle_side=True)
    cb = cpu_oracle_builds(sh, p, args.warmup, args.steps, args.cpu_stride, calibrate=True)
    v = cb["value"]
    print(json.dumps({"metric": METRIC, "value": v, "unit": "builds/s", "impl": "reference", "n_gpus": 0,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * cb["step_seconds"],
                      "ms_per_step_note": "wall time of one sampled step (the value is extrapolated from it)",
                      "extrapolated": True, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                      "config": bench_config(label, sh.nb, args.density, world),
                      "cpu_baseline": cb,
                      "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# DRAM bytes per LL|DL quartet of one C60 build (role kernels + scatter),
# from one ncu capture of this benchmark's own command (five builds, caches
# left as the program uses them): (280.5 GB read + 273.0 GB written) / 5 builds
# / 20,498,336 quartets
LLDL_DRAM_BYTES_PER_QUARTET = 5401.0


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    from hfcode_b200 import fock
    from hfcode_b200.csrc import gen_eri  # noqa: F401  (flop table lives beside the generator)
    label, mol, sh, p = workload(args.molecule, args.density)
    nb = sh.nb
    fb = fock.FockBuilder(sh)
    # cycle-1 set-up: Schwarz factors (not timed)
    f0 = np.zeros((nb, nb))
    fb.fock_build_initial_diag(f0, p, THR)
    dev = torch.device("cuda", local)
    P = torch.from_numpy(np.ascontiguousarray(p)).to(dev)
    F = torch.zeros((nb, nb), dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(fb.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        fb.fock_build_device(F.data_ptr(), P.data_ptr(), THR, THR, args.cutoff)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    n_launch0 = fb.launch_count()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    n_launch = fb.launch_count() - n_launch0  # this library's kernels in the timed steps
    total_ms = float(sum(times))
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = world * args.steps / (total_ms / 1000.0)
    st = fb.class_stats()
    n_pass = int(st["pass"].sum())
    # e2e through the reference-facing C ABI with host buffers (pinned, as
    # a caller that keeps its F and P in page-locked memory passes them)
    fh = torch.zeros((nb, nb), dtype=torch.float64, pin_memory=True).numpy()
    ph = torch.from_numpy(np.ascontiguousarray(p)).pin_memory().numpy()
    fb.fock_build_diag(fh, ph, THR)
    fb.fock_build_non_diag(fh, ph, THR)
    if dist:
        dist.barrier()
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fb.fock_build_diag(fh, ph, THR)
        fb.fock_build_non_diag(fh, ph, THR)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(sum(e2e_t))
    if dist:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * args.steps / e2e_s, "unit": "builds/s", "host_buffers": "pinned",
           "h2d_bytes_per_step": 2 * 2 * nb * nb * 8, "d2h_bytes_per_step": 2 * nb * nb * 8}
    # instrumented step: per-class kernel times for the roofline
    fb.set_timing(True)
    step()
    torch.cuda.synchronize()
    st = fb.class_stats()
    fb.set_timing(False)
    flops_tab = json.load(open(os.path.join(ROOT, "hfcode_b200", "csrc", "generated", "class_flops.json")))
    cls_flops = np.array([flops_tab[str(c)]["flops_prim"] * st["prim"][c] + flops_tab[str(c)]["flops_quartet"] *
                          st["pass"][c] for c in range(fock.NCLASS)], dtype=np.float64)
    top = int(np.argmax(st["ms"]))
    fp64_peak, fp32_peak = fock.measure_fma_peak()
    achieved = cls_flops[top] / (st["ms"][top] * 1e-3) / 1e12
    peak_tf = fp64_peak / 1e3
    # DRAM bytes per LL|DL quartet (role kernels + scatter) from one ncu
    # capture of this command on C60, times this build's LL|DL quartet count
    traffic = None
    if fock.CLASS_NAMES[top] == "LL|DL":
        traffic = LLDL_DRAM_BYTES_PER_QUARTET * float(st["pass"][top])
    # the same class seen from HBM: its measured DRAM bytes per build over
    # its time, against the measured copy bandwidth (fallback 6650 GB/s)
    hbm_peak, hbm_src = 6650.0, "fallback 6650 GB/s (no MEASURED_PEAKS.json)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            hbm_peak, hbm_src = float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        pass
    hbm_view = None
    if traffic:
        gbs = traffic / (st["ms"][top] * 1e-3) / 1e9
        hbm_view = {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                    "peak_source": hbm_src}
    roof = {"bound": "fp64", "kernel": f"class {fock.CLASS_NAMES[top]} (role kernels + k_scatter_staged)",
            "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s", "frac": achieved / peak_tf,
            "traffic": traffic, "traffic_unit": "bytes per build of the class",
            "traffic_source": "ncu capture of this C60 command (dram__bytes_read.sum + dram__bytes_write.sum of "
                              "the LL|DL role kernels and scatter, five builds): 5401 bytes per LL|DL quartet, "
                              "times this build's LL|DL quartet count",
            "hbm_view": hbm_view,
            "peak_source": "measured FP64 FMA-chain probe on this device (MEASURED_PEAKS.json has no FP64 figure)",
            "all_classes_tflops": float(cls_flops.sum() / (st["ms"].sum() * 1e-3) / 1e12),
            "class_ms": {fock.CLASS_NAMES[c]: round(float(st["ms"][c]), 3) for c in range(fock.NCLASS) if st["ms"][c] > 0},
            "class_tflops": {fock.CLASS_NAMES[c]: round(float(cls_flops[c] / (st["ms"][c] * 1e-3) / 1e12), 3)
                             for c in range(fock.NCLASS) if st["ms"][c] > 0},
            "class_quartets": {fock.CLASS_NAMES[c]: int(st["pass"][c]) for c in range(fock.NCLASS) if st["pass"][c] > 0},
            "class_prim_quartets": {fock.CLASS_NAMES[c]: int(st["prim"][c]) for c in range(fock.NCLASS) if st["prim"][c] > 0}}
    out = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if args.cutoff <= 0 else f"f64 + f32 below bound {args.cutoff:g}", "data": "synthetic",
           "config": bench_config(label, nb, args.density, world),
           "quartets_per_s": n_pass * value, "screened_in_quartets": n_pass,
           "e2e": e2e, "gpu_launches": n_launch, "roofline": roof,
           "fp64_peak_tflops": peak_tf, "fp32_peak_tflops": fp32_peak / 1e3,
           "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_mixed:
        out["mixed"] = mixed_study(fock, mol, sh, [float(x) for x in args.mixed_cutoffs.split(",")], dev)
    if rank == 0 and world == 1 and not args.no_serve:
        out["batching"] = batch_study(fock, dev)
        out["served"] = served_study(args.serve_jobs, args.serve_rate, 8, args.serve_plain)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_oracle_builds(sh, p, 1, 2, args.cpu_stride, calibrate=True)
    if rank == 0:
        print(json.dumps(out))
    fb.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
