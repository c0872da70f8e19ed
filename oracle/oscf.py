"""CPU oracle of the reference's direct-SCF protocol -- TEST INFRASTRUCTURE.

Only tests/, the golden-fixture script and bench.py's CPU legs use this; the
product package never imports it.  It restates direct_hartreefock.f90:1-234
around the oracle's own pieces, so that a converged energy from here shares
no arithmetic with the product (hfcode_b200):

  S, T, V        liboracle.so orc_one_electron (cmpt1e.f90, one_electron_terms.f90)
  G(P)           liboracle.so fock_build_* (the reference's three builders)
  E_nuc          nuclear_repulsion.f90:1-20, written out below
  eigensolve     numpy.linalg.eigh (LAPACK dsyevd) in the role of wrapper_dsyev
  DIIS solve     scipy LAPACK dsysv, as wrapper_dsysv (wrapper_dsygv.f90:55-78)

The protocol, with the reference lines it follows:
  :22-29    S^-1/2 = U diag(1/sqrt(s)) U^T from the eigenvectors of S
  :50-59    atomic-density guess, or :61-91 the core-Hamiltonian guess
  :98-121   cycle 1 initial_diag + non_diag; full builds while fullfock;
            otherwise diag(dP, thr) + non_diag(dP, thr*0.1) added to the
            previous F, with a full build forced after 15 incremental ones
  :123-131  E_elec = sum P (H + F) / 2
  :133-147  residual S^-1/2^T (FPS - SPF) S^-1/2 and the 8-deep histories
  :148-160  DIIS on at resmax < 0.3 (cycle >= 2); threshold drop to 1e-10
            with a forced full build at resmax < 0.005 (cycle >= 7)
  :161-199  DIIS: B_jk = <r_j, r_k>, diagonal x1.05 except the lowest-energy
            entry, rejected when max|c| >= 1.5
  :200-206  optional level shift, then the eigensolve of the extrapolated F
  :211-216  converged when |dE| < conve and max|dP| < conv (cycle > 1)
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np
import scipy.linalg

from oracle.pyoracle import Oracle

INTTHRESH = 1e-10   # molprops.f90:162
LOWTHRESH = 5e-7    # direct_hartreefock.f90:19
FDIFFFAC = 0.1
NDIIS = 8


def nuclear_repulsion(charges, coords) -> float:
    """nuclear_repulsion.f90:1-20: sum over atom pairs of Z_i Z_j / r_ij."""
    z = np.asarray(charges, dtype=np.float64)
    x = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    e = 0.0
    for i in range(len(z)):
        for j in range(i + 1, len(z)):
            e += z[i] * z[j] / math.sqrt(float(np.dot(x[i] - x[j], x[i] - x[j])))
    return e


def orthogonaliser(S: np.ndarray) -> np.ndarray:
    s, U = np.linalg.eigh(S)
    return U @ np.diag(1.0 / np.sqrt(s)) @ U.T


def core_guess(S, T, V, nocc: int) -> np.ndarray:
    """Core-Hamiltonian guess density (direct_hartreefock.f90:61-74)."""
    X = orthogonaliser(S)
    _, Cob = np.linalg.eigh(X @ (T + V) @ X.T)
    C = X @ Cob
    return 2.0 * C[:, :nocc] @ C[:, :nocc].T


class OracleSCF:
    """Direct RHF on the CPU oracle for one molecule and shell set."""

    def __init__(self, charges, coords, nocc: int, shells):
        self.charges = np.asarray(charges, dtype=np.float64)
        self.coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
        self.nocc = int(nocc)
        self.orc = Oracle(shells)
        self.nb = shells.nb
        self.S, self.T, self.V = self.orc.one_electron(self.charges, self.coords)
        self.enuc = nuclear_repulsion(self.charges, self.coords)

    def core_density(self) -> np.ndarray:
        return core_guess(self.S, self.T, self.V, self.nocc)

    def run(self, p_guess: Optional[np.ndarray] = None, maxiter: int = 60, conve: float = 5e-8,
            conv: float = 1e-5, levshft: Optional[float] = None, log=None):
        nb, nocc, orc = self.nb, self.nocc, self.orc
        S = self.S
        hcore = self.T + self.V
        X = orthogonaliser(S)
        resid_hist = np.full((NDIIS, nb, nb), 1000.0)
        fob_hist = np.zeros((NDIIS, nb, nb))
        e_hist = np.zeros(NDIIS)
        thresh = LOWTHRESH
        diis = False
        fullfock = True
        shift = None
        if levshft is not None:
            shift = np.zeros((nb, nb))
            shift[np.arange(nocc, nb), np.arange(nocc, nb)] = levshft
        cob = None
        if p_guess is None:
            _, cob = np.linalg.eigh(X @ hcore @ X.T)
            C = X @ cob
            p = 2.0 * C[:, :nocc] @ C[:, :nocc].T
            eelec = float(np.sum(p * hcore))
            use_shift = True
        else:
            p = np.array(p_guess, dtype=np.float64)
            eelec = 0.0
            use_shift = False
        pold = p.copy()
        f_prev = None
        nused = 0
        nfull = 0
        converged = False
        cycles = 0
        etot = eelec + self.enuc
        for it in range(1, maxiter + 1):
            cycles = it
            e_before = eelec
            f = hcore.copy()
            if fullfock and it == 1:
                orc.fock_build_initial_diag(f, p, thresh)
                orc.fock_build_non_diag(f, p, thresh)
                nfull = 0
            elif fullfock:
                orc.fock_build_diag(f, p, thresh)
                orc.fock_build_non_diag(f, p, thresh)
                fullfock = False
                nfull = 0
            else:
                dp = p - pold
                df = np.zeros((nb, nb))
                orc.fock_build_diag(df, dp, thresh)
                orc.fock_build_non_diag(df, dp, thresh * FDIFFFAC)
                f = f_prev + df
                nfull += 1
                if nfull == 15:
                    fullfock = True
            eelec = 0.5 * float(np.sum(p * (hcore + f)))
            de = eelec - e_before
            etot = eelec + self.enuc
            f_prev = f.copy()
            fob = X @ f @ X.T
            r = X.T @ (f @ p @ S - S @ p @ f) @ X
            resid_hist = np.roll(resid_hist, 1, axis=0)
            fob_hist = np.roll(fob_hist, 1, axis=0)
            e_hist = np.roll(e_hist, 1)
            resid_hist[0], fob_hist[0], e_hist[0] = r, fob, eelec
            resmax = float(np.max(np.abs(r)))
            if it >= 2 and resmax < 0.3 and not diis:
                diis = True
                use_shift = False
            if it >= 7 and thresh > INTTHRESH and resmax < 0.005:
                e_hist[:] = 2000.0
                nused = 0
                fullfock = True
                use_shift = False
                thresh = INTTHRESH
            if diis:
                nused = min(nused + 1, NDIIS)
                if nused > 1:
                    n = nused
                    B = np.zeros((n + 1, n + 1))
                    B[n, :n] = B[:n, n] = -1.0
                    for j in range(n):
                        for k in range(j + 1):
                            B[j, k] = B[k, j] = float(np.sum(resid_hist[j] * resid_hist[k]))
                    low = int(np.argmin(e_hist))
                    for j in range(n):
                        if j != low:
                            B[j, j] *= 1.05
                    rhs = np.zeros(n + 1)
                    rhs[n] = -1.0
                    c = scipy.linalg.lapack.dsysv(B, rhs.reshape(-1, 1), lower=0)[2][:, 0]
                    if np.max(np.abs(c[:n])) < 1.5:
                        fob = np.tensordot(c[:n], fob_hist[:n], axes=1)
                    else:
                        nused = 0
            if use_shift and shift is not None and cob is not None:
                fob = fob + cob @ shift @ cob.T
            _, cob = np.linalg.eigh(fob)
            C = X @ cob
            dpmax = float(np.max(np.abs(p - pold)))
            if log:
                log({"cycle": it, "etot": etot, "deltae": de, "deltap": dpmax, "thresh": thresh})
            if abs(de) < conve and dpmax < conv and it > 1:
                converged = True
                break
            pold = p
            p = 2.0 * C[:, :nocc] @ C[:, :nocc].T
        return {"energy": etot, "eelec": eelec, "enuc": self.enuc, "converged": converged, "cycles": cycles,
                "P": p, "F": f_prev}
