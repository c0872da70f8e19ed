"""Continuous-batching SCF server on one GPU.

The reference runs one RHF job per process (hf.f90).  This request loop
serves a stream of jobs on one B200:

* admission by device-memory footprint: a job is admitted when a slot is
  free and its estimated footprint (pair data, screening tables, quartet
  lists, scratch, F/P/G) fits the remaining budget; after the job's
  Schwarz pass the estimate is replaced by the handle's actual usage;
* each admitted job keeps its whole state resident on the device -- its own
  FockBuilder handle (screening tables, quartet lists, CUDA streams) and a
  device SCF job (density, Fock matrices, DIIS histories, S^-1/2; the
  library's C++ runs every cycle, include/hfgpu_scf.h) -- in a worker
  thread; the ctypes calls release the GIL, so concurrent jobs overlap on
  the GPU and no per-cycle work waits on Python;
* requests that arrive while others run wait in a FIFO and are admitted as
  slots and memory free up (continuous batching, not a batch barrier);
* metrics: jobs/s over the stream and per-job latency (arrival -> result)
  percentiles, plus queueing and service times.

Jobs run the mixed-precision form by default (FP32 for incremental-build
quartets whose screening bound is below `fp32_cutoff`), the FP64 form with
fp32_cutoff = 0.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import queue
import threading
import time
from typing import Dict, List, Optional

import numpy as np

from . import basis as basismod
from . import molecules, onee, scf
from .basis import Molecule, ShellSet


@dataclasses.dataclass
class Job:
    jid: int
    name: str
    mol: Molecule
    arrival: float                 # seconds from the start of the stream
    sh: Optional[ShellSet] = None
    p0: Optional[np.ndarray] = None
    footprint: int = 0
    admitted: float = 0.0
    finished: float = 0.0
    energy: float = float("nan")
    cycles: int = 0
    converged: bool = False
    error: str = ""


def make_stream(n_jobs: int, rate: float, seed: int = 20261203, max_alkane: int = 16, max_water: int = 20):
    """Seeded Poisson arrivals, uniform over CnH2n+2 (n = 1..max_alkane,
    all-anti) and (H2O)k (k = 1..max_water, rigid monomers at seeded random
    orientations, O-O >= 2.7 A)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    kinds = [("alkane", n) for n in range(1, max_alkane + 1)] + [("water", k) for k in range(1, max_water + 1)]
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        kind, n = kinds[int(rng.integers(len(kinds)))]
        if kind == "alkane":
            mol, name = molecules.alkane(n), f"C{n}H{2 * n + 2}"
        else:
            mol, name = molecules.water_cluster(n, np.random.default_rng(seed + 7919 * (j + 1))), f"(H2O){n}"
        jobs.append(Job(j, name, mol, t))
    return jobs


def estimate_footprint(sh: ShellSet, scratch_budget: int) -> int:
    """Upper-bound device bytes of one job before its Schwarz pass."""
    nb, nsh = sh.nb, sh.nsh
    npairs = nsh * (nsh + 1) // 2
    nprim = int(np.sum(sh.nzet[:, None] * sh.nzet[None, :])) // 2 + int(np.sum(sh.nzet ** 2))
    quartets = npairs * (npairs - 1) // 2 + npairs
    b = 3 * nb * nb * 8 + nsh * nsh * 8 + 2 * 7 * 8 * nprim + npairs * 200 + quartets * 8
    b += min(scratch_budget, quartets * 8 * 700)
    b += (13 + 2 * 8) * nb * nb * 8 + (8 << 20)  # device SCF state (hfgpu_scf_create) and its workspaces
    return int(b + (64 << 20))  # + CUDA context share / streams / tables


class Server:
    def __init__(self, hbm_budget: int, max_slots: int = 8, scratch_budget: int = 256 << 20,
                 fp32_cutoff: float = 1e-7, conve: float = 1e-8, conv: float = 1e-6, basis_name: str = "6-31G(d)",
                 graphs: bool = False, step: str = "device"):
        from . import fock  # loads the CUDA library; fails loudly without it
        self.fock = fock
        self.hbm_budget = hbm_budget
        self.max_slots = max_slots
        self.scratch_budget = scratch_budget
        self.fp32_cutoff = fp32_cutoff
        self.conve, self.conv = conve, conv
        # builds after the first as CUDA-graph replays; off by default: a
        # served SCF changes its thresholds four times in ~15 cycles, so each
        # job records four graphs for ~13 replays, and the recordings (taken
        # under the library's device lock) cost more than the launches they
        # save (measured 7.8 vs 11.9 jobs/s, 200 jobs, 8 slots)
        self.graphs = graphs
        # "device": the SCF cycle runs in the library's C++ with the job's
        # state on the GPU; "host": scf.direct_hartreefock (numpy/LAPACK
        # between builds, the state on the host)
        if step not in ("device", "host"):
            raise ValueError("step must be 'device' or 'host'")
        self.step = step
        self.basis = basismod.load_basis(basis_name)
        self.lock = threading.Condition()
        self.in_use = 0
        self.active = 0
        self.peak_in_use = 0
        self.peak_active = 0

    def warmup(self):
        """One tiny job per slot, all at once, before a stream: the library's
        per-process set-up (module loading, the pooled cuBLAS/cuSOLVER
        handles the device step borrows, the memory pool) happens here rather
        than in the first jobs' latencies."""
        jobs = [Job(-1 - k, "H2O", molecules.water_cluster(1, np.random.default_rng(k)), 0.0)
                for k in range(self.max_slots)]
        saved = (self.active, self.in_use, self.peak_active, self.peak_in_use)
        self._serve(jobs, realtime=False)
        self.active, self.in_use, self.peak_active, self.peak_in_use = saved

    def prepare(self, job: Job):
        job.sh = basismod.spread_basis(job.mol, self.basis)
        job.p0 = basismod.density_superposition(job.mol, self.basis, job.sh.nb)
        job.footprint = estimate_footprint(job.sh, self.scratch_budget)

    def _admit(self, job: Job):
        with self.lock:
            while not (self.active < self.max_slots and self.in_use + job.footprint <= self.hbm_budget):
                self.lock.wait()
            self.active += 1
            self.in_use += job.footprint
            self.peak_active = max(self.peak_active, self.active)
            self.peak_in_use = max(self.peak_in_use, self.in_use)

    def _release(self, amount: int):
        with self.lock:
            self.active -= 1
            self.in_use -= amount
            self.lock.notify_all()

    def _adjust(self, job: Job, actual: int):
        with self.lock:
            self.in_use += actual - job.footprint
            job.footprint = actual
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            self.lock.notify_all()

    def run_job(self, job: Job, t0: float):
        if self.step == "device":
            return self._run_job_device(job, t0)
        fb = None
        try:
            fb = self.fock.FockBuilder(job.sh, scratch_budget=self.scratch_budget)

            class Tracked:
                """Forwards the builder calls; updates the admission account
                with the handle's real usage after the Schwarz pass."""

                def __init__(s, inner):
                    s.inner = inner

                def fock_build_initial_diag(s, f, p, thr):
                    s.inner.fock_build_initial_diag(f, p, thr)
                    self._adjust(job, s.inner.device_bytes() + (64 << 20))

                def __getattr__(s, name):
                    return getattr(s.inner, name)

            ints = onee.one_electron(job.mol, job.sh, gpu=True)
            r = scf.direct_hartreefock(job.mol, job.sh, Tracked(fb), p_guess=job.p0, conve=self.conve,
                                       conv=self.conv, maxiter=60, ints=ints, fp32_cutoff=self.fp32_cutoff,
                                       graph=self.graphs)
            job.energy, job.cycles, job.converged = r.energy, r.cycles, r.converged
        except Exception as e:  # the job fails, the server keeps serving
            job.error = f"{type(e).__name__}: {e}"
        finally:
            if fb is not None:
                fb.close()
            job.finished = time.perf_counter() - t0
            self._release(job.footprint)

    def _run_job_device(self, job: Job, t0: float):
        fb = dj = None
        try:
            fb = self.fock.FockBuilder(job.sh, scratch_budget=self.scratch_budget)
            S, T, V = onee.one_electron(job.mol, job.sh, gpu=True)
            dj = self.fock.DeviceSCFJob(fb, job.mol.nocc, job.mol.nuclear_repulsion(), S, T + V, job.p0)
            kw = dict(conve=self.conve, conv=self.conv, fp32_cutoff=self.fp32_cutoff)
            dj.run(maxiter=1, **kw)  # cycle 1: the Schwarz pass sizes the handle's lists and scratch
            self._adjust(job, fb.device_bytes() + dj.device_bytes() + (64 << 20))
            r = dj.run(maxiter=60, **kw)
            job.energy, job.cycles, job.converged = r["energy"], r["cycles"], bool(r["converged"])
        except Exception as e:  # the job fails, the server keeps serving
            job.error = f"{type(e).__name__}: {e}"
        finally:
            if dj is not None:
                dj.close()
            if fb is not None:
                fb.close()
            job.finished = time.perf_counter() - t0
            self._release(job.footprint)

    @property
    def blas_threads(self) -> int:
        """Host BLAS/LAPACK threads: the cores shared among the slots.  Every
        job's SCF step calls LAPACK from its own thread; letting each call
        use all cores oversubscribes the host (measured 3.4 -> 10.7 jobs/s
        on a 16-core host with 8 slots when limited to 2 threads)."""
        return max(1, (os.cpu_count() or 1) // self.max_slots)

    def serve(self, jobs: List[Job], realtime: bool = True) -> Dict:
        """Runs the stream; each job is released at its arrival time (or all
        at once with realtime=False) and admitted FIFO."""
        from threadpoolctl import threadpool_limits
        with threadpool_limits(limits=self.blas_threads):
            return self._serve(jobs, realtime)

    def _serve(self, jobs: List[Job], realtime: bool) -> Dict:
        for j in jobs:
            self.prepare(j)
        t0 = time.perf_counter()
        threads = []
        for j in sorted(jobs, key=lambda x: x.arrival):
            if realtime:
                wait = j.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            else:
                j.arrival = time.perf_counter() - t0
            if j.footprint > self.hbm_budget:
                j.error = "footprint exceeds the server's HBM budget"
                j.admitted = j.finished = time.perf_counter() - t0
                continue
            self._admit(j)  # FIFO: the next arrival waits behind this one
            j.admitted = time.perf_counter() - t0
            th = threading.Thread(target=self.run_job, args=(j, t0), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        makespan = max(j.finished for j in jobs) - min(j.arrival for j in jobs)
        lat = np.array([j.finished - j.arrival for j in jobs]) * 1e3
        svc = np.array([j.finished - j.admitted for j in jobs]) * 1e3
        que = np.array([j.admitted - j.arrival for j in jobs]) * 1e3
        return {"jobs": len(jobs), "jobs_per_s": len(jobs) / makespan, "makespan_s": makespan,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                               "mean": float(lat.mean())},
                "service_ms": {"p50": float(np.percentile(svc, 50)), "p99": float(np.percentile(svc, 99))},
                "queue_ms": {"p50": float(np.percentile(que, 50)), "p99": float(np.percentile(que, 99))},
                "failed": sum(1 for j in jobs if j.error), "not_converged": sum(1 for j in jobs if not j.converged),
                "errors": sorted({j.error for j in jobs if j.error})[:5],
                "peak_active": self.peak_active, "peak_hbm_bytes": self.peak_in_use,
                "max_slots": self.max_slots, "hbm_budget": self.hbm_budget, "fp32_cutoff": self.fp32_cutoff}


def serve_sequential(jobs: List[Job], server: Server) -> Dict:
    """The plain per-job form: one job at a time on the GPU, same protocol."""
    from threadpoolctl import threadpool_limits
    with threadpool_limits(limits=server.blas_threads):
        return _serve_sequential(jobs, server)


def _serve_sequential(jobs: List[Job], server: Server) -> Dict:
    for j in jobs:
        server.prepare(j)
    t0 = time.perf_counter()
    for j in sorted(jobs, key=lambda x: x.arrival):
        now = time.perf_counter() - t0
        j.admitted = max(now, j.arrival)
        if j.arrival > now:
            time.sleep(j.arrival - now)
        server._admit(j)
        server.run_job(j, t0)
    makespan = max(j.finished for j in jobs) - min(j.arrival for j in jobs)
    lat = np.array([j.finished - j.arrival for j in jobs]) * 1e3
    return {"jobs": len(jobs), "jobs_per_s": len(jobs) / makespan, "makespan_s": makespan,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "mean": float(lat.mean())}}


def main():
    ap = argparse.ArgumentParser(description="Continuous-batching RHF server on one GPU")
    ap.add_argument("--jobs", type=int, default=1000)
    ap.add_argument("--rate", type=float, default=20.0, help="Poisson arrival rate, jobs/s")
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--hbm-gb", type=float, default=64.0)
    ap.add_argument("--fp32-cutoff", type=float, default=1e-7)
    ap.add_argument("--sequential", action="store_true", help="also run the plain per-job form")
    ap.add_argument("--graphs", action="store_true", help="host step: builds after the first as graph replays")
    ap.add_argument("--step", default="device", choices=["device", "host"])
    args = ap.parse_args()
    srv = Server(int(args.hbm_gb * (1 << 30)), args.slots, fp32_cutoff=args.fp32_cutoff,
                 graphs=args.graphs, step=args.step)
    jobs = make_stream(args.jobs, args.rate)
    srv.warmup()
    out = {"served": srv.serve(jobs)}
    if args.sequential:
        seq = make_stream(args.jobs, args.rate)
        out["sequential"] = serve_sequential(seq, Server(int(args.hbm_gb * (1 << 30)), 1,
                                                        fp32_cutoff=args.fp32_cutoff,
                                                        graphs=args.graphs, step=args.step))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
