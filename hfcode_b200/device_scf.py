"""Device-resident RHF: the reference's SCF protocol with every per-cycle array
on the GPU and each cycle replayed as one CUDA graph.

The host driver (scf.direct_hartreefock) restates direct_hartreefock.f90 with
numpy/LAPACK between Fock builds.  Here the whole cycle stays on the device:

  Fock build (hfgpu_fock_build_device_on: full, or incremental on dP with
  thr and thr*fdifffac, mixed below `fp32_cutoff`)  ->  E_elec = 1/2 sum P(H+F)
  (direct_hartreefock.f90:123-131)  ->  orthogonalised F and the commutator
  residual X^T (FPS - SPF) X  ->  DIIS over up to 8 vectors with the diagonal
  scaled by 1.05 except the lowest-energy entry, rejected when max|c| >= 1.5
  (:133-199; the bordered system is solved by hfgpu_small_solve)  ->  the new
  density  ->  max|dP|.

The reference diagonalises the orthogonal Fock matrix (dsyev, :204) and
builds P from the occupied eigenvectors.  A dense eigensolver cannot be
recorded in a CUDA graph (cuSOLVER's syevd synchronises with the host), so
the occupied projector is formed by second-order spectral projection
(SP2: A. M. N. Niklasson, Phys. Rev. B 66, 155115 (2002)): starting from the
Gershgorin-scaled Fock matrix, each step replaces X by X^2 or 2X - X^2,
whichever keeps trace(X) nearer the number of occupied orbitals.  For a
closed-shell system with a HOMO-LUMO gap this converges quadratically to the
same projector the eigenvectors give, using FP64 matrix products only.

The protocol's decisions (DIIS start, threshold drop, full vs incremental
build, convergence) are made on the device where they depend on this cycle's
numbers; the host reads five scalars per cycle and picks the next graph:
(full | incremental) x (loose | tight threshold), plus the first cycle, whose
Fock build (the Schwarz pass) runs through the host interface.
"""
from __future__ import annotations

import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import onee
from .basis import Molecule, ShellSet
from .scf import INTTHRESH, SCFResult

NDIIS = 8


class DeviceSCF:
    """One SCF instance's device state; `run` is the protocol."""

    def __init__(self, mol: Molecule, sh: ShellSet, builder, ints=None, sp2_steps: int = 64,
                 graphs: bool = True, device: str = "cuda"):
        import torch
        self.torch = torch
        self.mol, self.sh, self.fb = mol, sh, builder
        self.nb = sh.nb
        self.nocc = mol.nocc
        self.sp2_steps = sp2_steps
        self.graphs = graphs
        self.dev = torch.device(device)
        S, T, V = ints if ints is not None else onee.one_electron(mol, sh, gpu=True)
        e, U = np.linalg.eigh(S)
        X = (U / np.sqrt(e)) @ U.T  # S^-1/2 (direct_hartreefock.f90:22-29), once per job
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=self.dev)
        nb = self.nb
        self.S, self.X, self.H = t(S), t(0.5 * (X + X.T)), t(T + V)
        z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=self.dev)
        self.P, self.Pold, self.Pnew = z(nb, nb), z(nb, nb), z(nb, nb)
        self.F, self.Fold, self.dF = z(nb, nb), z(nb, nb), z(nb, nb)
        self.R, self.FO = z(NDIIS, nb, nb), z(NDIIS, nb, nb)
        self.eo = z(NDIIS)
        self.n = torch.zeros((), dtype=torch.int64, device=self.dev)      # nusediis
        self.diis = torch.zeros((), dtype=torch.bool, device=self.dev)
        self.it = torch.zeros((), dtype=torch.int64, device=self.dev)     # cycle number
        self.A = z(NDIIS + 1, NDIIS + 1)
        self.rhs = z(NDIIS + 1)
        self.rhs0 = z(NDIIS + 1)
        self.rhs0[NDIIS] = -1.0  # the Lagrange row of the DIIS system
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.out = z(5)  # eelec, resmax, deltap, threshold-drop flag, nusediis
        self.idx = torch.arange(NDIIS, device=self.dev)
        self._graphs: Dict[tuple, object] = {}
        self.enuc = mol.nuclear_repulsion()

    # ------------------------------------------------------------ one cycle
    def _build(self, kind: str, thr: float, fdifffac: float, cut: float):
        """Fock matrix of this cycle on the current stream."""
        torch = self.torch
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        if kind == "full":
            self.F.copy_(self.H)
            self.fb.fock_build_device_on(self.F.data_ptr(), self.P.data_ptr(), thr, thr, 0.0, stream)
        elif kind == "delta":
            dP = self.P - self.Pold
            self.dF.zero_()
            self.fb.fock_build_device_on(self.dF.data_ptr(), dP.data_ptr(), thr, thr * fdifffac, cut, stream)
            torch.add(self.Fold, self.dF, out=self.F)
        # kind "first": F was filled through the host interface

    def _post(self, loose: bool):
        """Everything after the Fock build: energy, residual, DIIS, density."""
        torch = self.torch
        S, X, H, P, F = self.S, self.X, self.H, self.P, self.F
        eelec = 0.5 * torch.sum(P * (H + F))
        fob = X @ F @ X
        comm = F @ P @ S
        comm = comm - comm.T  # S P F = (F P S)^T for symmetric F, P, S
        resid = X @ comm @ X
        resmax = resid.abs().max()
        # history, newest first (direct_hartreefock.f90:133-145)
        self.R[1:] = self.R[:-1].clone()
        self.FO[1:] = self.FO[:-1].clone()
        self.eo[1:] = self.eo[:-1].clone()
        self.R[0] = resid
        self.FO[0] = fob
        self.eo[0] = eelec
        self.diis |= (self.it >= 2) & (resmax < 0.3)
        drop = (self.it >= 7) & (resmax < 0.005) if loose else torch.zeros((), dtype=torch.bool, device=self.dev)
        self.eo.copy_(torch.where(drop, torch.full_like(self.eo, 2000.0), self.eo))
        n = torch.where(drop, torch.zeros_like(self.n), self.n)
        n = torch.where(self.diis, torch.clamp(n + 1, max=NDIIS), n)
        # bordered DIIS system with the Lagrange row last; unused slots are
        # identity rows so their coefficients come out zero
        valid = self.idx < n
        vf = valid.to(torch.float64)
        B = torch.einsum("jab,kab->jk", self.R, self.R) * torch.outer(vf, vf)
        lowest = torch.argmin(self.eo)  # over the whole history, as the reference does
        scale = torch.where(valid & (self.idx != lowest), 1.05, 1.0).to(torch.float64)
        eye8 = torch.eye(NDIIS, dtype=torch.float64, device=self.dev)
        B = B * (1.0 - eye8) + torch.diag(B.diagonal() * scale) + torch.diag(1.0 - vf)
        self.A.zero_()
        self.A[:NDIIS, :NDIIS] = B
        self.A[NDIIS, :NDIIS] = -vf
        self.A[:NDIIS, NDIIS] = -vf
        self.rhs.copy_(self.rhs0)
        from .fock import small_solve
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        small_solve(self.A.data_ptr(), self.rhs.data_ptr(), NDIIS + 1, self.status.data_ptr(), stream)
        c = self.rhs[:NDIIS]
        use = n > 1
        ok = (self.status[0] == 1) & (c.abs().max() < 1.5)
        fob = torch.where(use & ok, torch.einsum("j,jab->ab", c, self.FO), fob)
        self.n.copy_(torch.where(use & ~ok, torch.zeros_like(n), n))
        # density: occupied projector of fob by SP2, back to the AO basis
        D = self._sp2(fob)
        Pn = 2.0 * (X @ D @ X)
        self.Pnew.copy_(0.5 * (Pn + Pn.T))
        deltap = (P - self.Pold).abs().max()
        self.Fold.copy_(F)
        self.out[0] = eelec
        self.out[1] = resmax
        self.out[2] = deltap
        self.out[3] = drop.to(torch.float64)
        self.out[4] = self.n.to(torch.float64)

    def _sp2(self, F):
        torch = self.torch
        nb = self.nb
        eye = torch.eye(nb, dtype=torch.float64, device=self.dev)
        off = F.abs().sum(dim=1) - F.diagonal().abs()
        emin = (F.diagonal() - off).min()
        emax = (F.diagonal() + off).max()
        Xk = (emax * eye - F) / (emax - emin)
        nocc = float(self.nocc)
        for _ in range(self.sp2_steps):
            X2 = Xk @ Xk
            tr, tr2 = Xk.diagonal().sum(), X2.diagonal().sum()
            Xk = torch.where(torch.abs(tr2 - nocc) < torch.abs(2.0 * tr - tr2 - nocc), X2, 2.0 * Xk - X2)
        return Xk

    def _cycle(self, kind: str, thr: float, fdifffac: float, cut: float, loose: bool):
        torch = self.torch
        key = (kind, thr, fdifffac, cut, loose)
        if not self.graphs:
            self._build(kind, thr, fdifffac, cut)
            self._post(loose)
            return
        g = self._graphs.get(key)
        if g is None:
            # the first cycle of a kind runs eagerly (which also warms up the
            # libraries) and is then recorded, without running it again, for
            # the later cycles of that kind
            self._build(kind, thr, fdifffac, cut)
            self._post(loose)
            from .fock import DEVICE_LOCK
            g = torch.cuda.CUDAGraph()
            with DEVICE_LOCK, torch.cuda.graph(g, capture_error_mode="thread_local"):
                self._build(kind, thr, fdifffac, cut)
                self._post(loose)
            self._graphs[key] = g
            return
        g.replay()

    # ------------------------------------------------------------ protocol
    def run(self, p_guess: np.ndarray, maxiter: int = 25, conv: float = 1e-5, conve: float = 5e-8,
            lowthresh: float = 5e-7, fdifffac: float = 0.1, fp32_cutoff: float = 0.0,
            log: Optional[Callable] = None) -> SCFResult:
        """direct_hartreefock.f90:93-223 with the per-cycle work on the device
        (see the module docstring); same arguments as scf.direct_hartreefock."""
        torch = self.torch
        nb = self.nb
        self.P.copy_(torch.as_tensor(np.ascontiguousarray(p_guess), dtype=torch.float64, device=self.dev))
        self.Pold.copy_(self.P)
        for t in (self.R, self.FO, self.eo, self.n, self.diis):
            t.zero_()
        fullfock, thresh, nfull, eelec = True, lowthresh, 0, 0.0
        hist: List[Dict] = []
        converged = False
        for it in range(1, maxiter + 1):
            t0 = time.perf_counter()
            self.it.fill_(it)
            eeold = eelec
            loose = thresh > INTTHRESH
            if fullfock and it == 1:
                # cycle 1: the Schwarz pass goes through the host interface
                f = (self.H.cpu().numpy()).copy()
                p = self.P.cpu().numpy()
                self.fb.fock_build_initial_diag(f, p, thresh)
                self.fb.fock_build_non_diag(f, p, thresh)
                self.F.copy_(torch.as_tensor(f, device=self.dev))
                kind = "first"
                self._build("first", thresh, fdifffac, 0.0)
                self._post(loose)  # eager: cycle 1 runs once
                nfull = 0
            else:
                if fullfock:
                    kind = "full"
                    fullfock = False
                    nfull = 0
                else:
                    kind = "delta"
                    nfull += 1
                    if nfull == 15:
                        fullfock = True
                self._cycle(kind, thresh, fdifffac, fp32_cutoff if kind == "delta" else 0.0, loose)
            eelec, resmax, deltap, drop, _ = (float(x) for x in self.out.cpu())
            deltae = eelec - eeold
            if drop > 0.5:  # direct_hartreefock.f90:152-160
                fullfock = True
                thresh = INTTHRESH
            hist.append({"cycle": it, "etot": eelec + self.enuc, "deltae": deltae, "deltap": deltap, "kind": kind,
                         "thresh": thresh, "t_cycle": time.perf_counter() - t0})
            if log:
                log(hist[-1])
            if abs(deltae) < conve and deltap < conv and it > 1:
                converged = True
                break
            self.Pold.copy_(self.P)
            self.P.copy_(self.Pnew)
        return SCFResult(energy=eelec + self.enuc, eelec=eelec, enuc=self.enuc, converged=converged,
                         cycles=len(hist), P=self.P.cpu().numpy(), F=self.Fold.cpu().numpy(),
                         eigs=np.zeros(nb), history=hist)
