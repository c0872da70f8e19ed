"""Direct RHF driver: the reference's SCF protocol around the Fock builder.

Restates direct_hartreefock.f90:1-234 on the host in FP64 (numpy/LAPACK), so
that the Fock builds it calls -- the GPU builder or the CPU oracle, both with
the fock_build_initial_diag / fock_build_diag / fock_build_non_diag
interface -- can be compared at the level of converged energies:

* S^-1/2 from the eigenvectors of S (:22-29); guess from atomic densities
  (:50-59) or the core Hamiltonian (:61-91);
* cycle 1: fock_build_initial_diag + fock_build_non_diag; the next cycle and
  every cycle with `fullfock` set: fock_build_diag + fock_build_non_diag;
  otherwise the incremental build on dP = P - Pold with thr and thr*fdifffac
  (:98-121), forced full every 15th incremental cycle;
* E_elec = 1/2 sum P (H + F) (:123-131); DIIS on the orthogonalised
  commutator with up to 8 vectors, the diagonal scaled by 1.05 except for the
  lowest-energy entry, rejected when max |c| >= 1.5 (:133-199);
* threshold drop to 1e-10 with a forced full build once resmax < 0.005
  after cycle 7 (:152-160); optional level shift (:200-203);
* convergence |dE| < conve and max |dP| < conv (:211-216).

`conve` and `conv` default to the reference's 5e-8 / 1e-5; parity studies
tighten them.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable, Dict, List, Optional

import numpy as np
import scipy.linalg

from . import onee
from .basis import Molecule, ShellSet

INTTHRESH = 1e-10  # molprops.f90:162


@dataclasses.dataclass
class SCFResult:
    energy: float
    eelec: float
    enuc: float
    converged: bool
    cycles: int
    P: np.ndarray
    F: np.ndarray
    eigs: np.ndarray
    history: List[Dict]


def dsysv(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """wrapper_dsysv (wrapper_dsygv.f90:55-78): symmetric indefinite solve."""
    lu, piv, x, info = scipy.linalg.lapack.dsysv(a, b.reshape(-1, 1), lower=0)
    return x[:, 0]


def direct_hartreefock(mol: Molecule, sh: ShellSet, builder, p_guess: Optional[np.ndarray] = None,
                       maxiter: int = 25, conv: float = 1e-5, conve: float = 5e-8,
                       lowthresh: float = 5e-7, fdifffac: float = 0.1, ndiis: int = 8,
                       levshft: Optional[float] = None, ints=None, log: Optional[Callable] = None,
                       fp32_cutoff: float = 0.0, graph: bool = False) -> SCFResult:
    """Runs the reference's direct SCF protocol with `builder`.

    fp32_cutoff > 0 selects the mixed-precision form for the incremental
    (delta-P) builds: quartets whose screening bound on dP falls below the
    cutoff are evaluated in FP32 by builder.fock_build_non_diag_mixed; full
    builds, accumulation, DIIS, the eigensolve and the energy stay FP64.

    graph=True runs every build after the first as one CUDA-graph replay
    (builder.fock_build_graph: diag + non-diag fused, with the same
    thresholds and arithmetic as the two separate calls)."""
    nb = sh.nb
    nocc = mol.nocc
    S, T, V = ints if ints is not None else onee.one_electron(mol, sh)
    e, U = np.linalg.eigh(S)
    sminhalf = (U / np.sqrt(e)) @ U.T
    hcore = T + V
    unuc = mol.nuclear_repulsion()
    resido = np.full((ndiis, nb, nb), 1000.0)
    fold = np.zeros((ndiis, nb, nb))
    eo = np.zeros(ndiis)
    diis = False
    fullfock = True
    eelec = 0.0
    thresh = lowthresh
    shftmat = None
    cmatob = None
    if levshft is not None:
        shftmat = np.zeros((nb, nb))
        for k in range(nocc, nb):
            shftmat[k, k] = levshft
    if p_guess is not None:
        p = np.array(p_guess, dtype=np.float64)
        uselevshft = False
    else:
        fob = sminhalf @ hcore @ sminhalf.T
        _, cmatob = np.linalg.eigh(fob)
        cmat = sminhalf @ cmatob
        p = 2.0 * cmat[:, :nocc] @ cmat[:, :nocc].T
        eelec = float(np.sum(p * hcore))
        uselevshft = True
    pold = p.copy()
    nusediis = 0
    nfull = 0
    faobold = None
    hist = []
    converged = False
    eigs = np.zeros(nb)
    t_start = time.perf_counter()
    for it in range(1, maxiter + 1):
        t0 = time.perf_counter()
        f = hcore.copy()
        eeold = eelec
        if fullfock and it == 1:
            builder.fock_build_initial_diag(f, p, thresh)
            builder.fock_build_non_diag(f, p, thresh)
            nfull = 0
            kind = "initial"
        elif fullfock:
            if graph:
                builder.fock_build_graph(f, p, thresh, thresh, 0.0)
            else:
                builder.fock_build_diag(f, p, thresh)
                builder.fock_build_non_diag(f, p, thresh)
            fullfock = False
            nfull = 0
            kind = "full"
        else:
            delp = p - pold
            delf = np.zeros((nb, nb))
            if graph:
                builder.fock_build_graph(delf, delp, thresh, thresh * fdifffac, fp32_cutoff)
            else:
                builder.fock_build_diag(delf, delp, thresh)
                if fp32_cutoff > 0.0:
                    builder.fock_build_non_diag_mixed(delf, delp, thresh * fdifffac, fp32_cutoff)
                else:
                    builder.fock_build_non_diag(delf, delp, thresh * fdifffac)
            f = faobold + delf
            nfull += 1
            if nfull == 15:
                fullfock = True
            kind = "delta"
        t_build = time.perf_counter() - t0
        eelec = 0.5 * float(np.sum(p * (hcore + f)))
        deltae = eelec - eeold
        etot = eelec + unuc
        faobold = f.copy()
        fob = sminhalf @ f @ sminhalf.T
        comm = f @ p @ S - S @ p @ f
        resid = sminhalf.T @ comm @ sminhalf
        resido[1:] = resido[:-1].copy()
        fold[1:] = fold[:-1].copy()
        eo[1:] = eo[:-1].copy()
        resido[0] = resid
        fold[0] = fob
        eo[0] = eelec
        resmax = float(np.max(np.abs(resid)))
        if it >= 2 and resmax < 0.3 and not diis:
            diis = True
            uselevshft = False
        if it >= 7 and thresh > INTTHRESH and resmax < 0.005:
            eo[:] = 2000.0
            nusediis = 0
            fullfock = True
            uselevshft = False
            thresh = INTTHRESH
        if diis:
            nusediis = min(nusediis + 1, ndiis)
            if nusediis > 1:
                n = nusediis
                bmat = np.zeros((n + 1, n + 1))
                bmat[n, :] = -1.0
                bmat[:, n] = -1.0
                bmat[n, n] = 0.0
                vecb = np.zeros(n + 1)
                vecb[n] = -1.0
                for j in range(n):
                    for k in range(j + 1):
                        bmat[j, k] = bmat[k, j] = float(np.sum(resido[j] * resido[k]))
                ii = int(np.argmin(eo))
                for j in range(n):
                    if j != ii:
                        bmat[j, j] *= 1.05
                solb = dsysv(bmat, vecb)
                if np.max(np.abs(solb[:n])) < 1.5:
                    fob = np.tensordot(solb[:n], fold[:n], axes=1)
                else:
                    nusediis = 0
        if uselevshft and shftmat is not None and cmatob is not None:
            fob = fob + cmatob @ shftmat @ cmatob.T
        eigs, cmatob = np.linalg.eigh(fob)
        cmat = sminhalf @ cmatob
        deltap = float(np.max(np.abs(p - pold)))
        hist.append({"cycle": it, "etot": etot, "deltae": deltae, "deltap": deltap, "kind": kind,
                     "thresh": thresh, "t_build": t_build, "t_cycle": time.perf_counter() - t0})
        if log:
            log(hist[-1])
        if abs(deltae) < conve and deltap < conv and it > 1:
            converged = True
            break
        pold = p
        p = 2.0 * cmat[:, :nocc] @ cmat[:, :nocc].T
    return SCFResult(energy=eelec + unuc, eelec=eelec, enuc=unuc, converged=converged, cycles=len(hist),
                     P=p, F=faobold, eigs=eigs, history=hist)


def device_hartreefock(mol: Molecule, sh: ShellSet, builder, p_guess: Optional[np.ndarray] = None,
                       maxiter: int = 25, conv: float = 1e-5, conve: float = 5e-8, fp32_cutoff: float = 0.0,
                       levshft: Optional[float] = None, ints=None) -> SCFResult:
    """The same protocol with the job's state on the GPU (fock.DeviceSCFJob):
    S^-1/2, the densities, Fock matrices and DIIS histories stay in device
    memory and every cycle runs from the library's C++ on the builder's
    stream; the host only starts the run and reads the result.  S, T, V come
    from the GPU one-electron integrals unless `ints` is given."""
    from . import fock
    S, T, V = ints if ints is not None else onee.one_electron(mol, sh, gpu=True)
    job = fock.DeviceSCFJob(builder, mol.nocc, mol.nuclear_repulsion(), S, T + V, p_guess)
    try:
        r = job.run(maxiter=maxiter, conv=conv, conve=conve, fp32_cutoff=fp32_cutoff,
                    levshft=levshft if levshft is not None else 0.0)
        P, F, eigs = job.get()
    finally:
        job.close()
    return SCFResult(energy=r["energy"], eelec=r["eelec"], enuc=r["energy"] - r["eelec"],
                     converged=bool(r["converged"]), cycles=r["cycles"], P=P, F=F, eigs=eigs,
                     history=[{"full_builds": r["full_builds"], "delta_builds": r["delta_builds"],
                               "deltae": r["deltae"], "deltap": r["deltap"]}])
