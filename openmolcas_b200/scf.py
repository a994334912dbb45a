"""Closed-shell SCF iteration over the Cholesky J/K build.

The caller loop around ``CHO_LK_SCF``: the reference's SCF program builds the
two-electron Fock matrix from Cholesky vectors in ``ChoSCF_Drv``
(``scf/choscf_drv.F90:15``, ``CHO_LK_SCF`` at :208) for the density of the
occupied orbitals, and iterates Roothaan steps with DIIS until the energy and
the density converge.  The energy is the one the reference prints as E_SCF
(``scf/prfin0.F90:147``): one-electron energy tr(D h) + two-electron energy
1/2 tr(D J) - 1/4 tr(D K) + nuclear repulsion, D = 2 C_occ C_occ^T.

Here the two-electron part is ``jk(C)``: J and K of D = C C^T, by default the
device build ``MolGpu.cho_jk`` (FP64) over vectors from ``MolGpu.cho_drv``.
The one-electron matrices h and S come from the caller (the reference reads
them from Seward's one-electron file).  Every matrix lives on one torch
device; the iteration is O(nbf^3) dense algebra per step (eigendecomposition,
DIIS extrapolation) next to the J/K build.

Restated with our own choices: core-Hamiltonian guess unless orbitals are
given, canonical orthogonalisation dropping overlap eigenvalues below
``lindep``, Pulay DIIS on the orthogonalised commutator FDS - SDF.
"""
from __future__ import annotations

from typing import Callable, Optional

import torch


def _orthogonaliser(S: torch.Tensor, lindep: float) -> torch.Tensor:
    s, U = torch.linalg.eigh(S)
    keep = s > lindep
    return U[:, keep] / torch.sqrt(s[keep])[None, :]


def rhf(jk: Callable[[torch.Tensor], tuple], h: torch.Tensor, S: torch.Tensor, nocc: int, enuc: float,
        C0: Optional[torch.Tensor] = None, e_conv: float = 1e-10, d_conv: float = 1e-8, maxiter: int = 100,
        ndiis: int = 8, lindep: float = 1e-9) -> dict:
    """Closed-shell SCF.  jk(C) returns (J, K) of D = C C^T (nbf x nbf).

    Returns dict(energy, C (nbf x nmo), eps (nmo), niter, converged, history):
    ``energy`` is E_SCF of the last density, ``history`` the energy per
    iteration.  Converged when the energy change is below ``e_conv`` and the
    largest element of the orthogonalised commutator below ``d_conv``.
    Raises ValueError when nocc exceeds the orbitals left after dropping
    near-linear dependencies or maxiter < 1."""
    if maxiter < 1:
        raise ValueError("rhf: maxiter must be >= 1")
    dev, dt = h.device, torch.float64
    h = h.to(dev, dt)
    S = S.to(dev, dt)
    X = _orthogonaliser(S, lindep)
    if not 0 < nocc <= X.shape[1]:
        raise ValueError(f"rhf: {nocc} occupied orbitals, {X.shape[1]} linearly independent functions")

    def diag(F):
        eps, Ct = torch.linalg.eigh(X.T @ F @ X)
        return eps, X @ Ct

    if C0 is None:
        eps, C = diag(h)
        Cocc = C[:, :nocc]
    else:
        Cocc = C0.to(dev, dt)[:, :nocc]
    fock_hist, err_hist, energies = [], [], []
    e_old = None
    converged = False
    eps = C = None
    for it in range(1, maxiter + 1):
        D = 2.0 * Cocc @ Cocc.T
        J, K = jk(Cocc * (2.0 ** 0.5))
        J = J.to(dev, dt)
        K = K.to(dev, dt)
        F = h + J - 0.5 * K
        E = float(torch.sum(D * h) + 0.5 * torch.sum(D * J) - 0.25 * torch.sum(D * K)) + enuc
        energies.append(E)
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        emax = float(err.abs().max())
        if e_old is not None and abs(E - e_old) < e_conv and emax < d_conv:
            converged = True
            eps, C = diag(F)
            break
        e_old = E
        fock_hist.append(F)
        err_hist.append(err)
        del fock_hist[:-ndiis], err_hist[:-ndiis]
        n = len(fock_hist)
        if n > 1:
            Bm = torch.empty((n + 1, n + 1), dtype=dt, device=dev)
            for i in range(n):
                for j in range(n):
                    Bm[i, j] = torch.sum(err_hist[i] * err_hist[j])
            Bm[n, :n] = -1.0
            Bm[:n, n] = -1.0
            Bm[n, n] = 0.0
            rhs = torch.zeros(n + 1, dtype=dt, device=dev)
            rhs[n] = -1.0
            try:
                c = torch.linalg.solve(Bm, rhs)[:n]
                F = sum(ci * Fi for ci, Fi in zip(c, fock_hist))
            except RuntimeError:  # singular subspace: restart it from the newest Fock matrix
                del fock_hist[:-1], err_hist[:-1]
        eps, C = diag(F)
        Cocc = C[:, :nocc]
    return dict(energy=energies[-1], C=C, eps=eps, niter=len(energies), converged=converged, history=energies)


def uhf(jk: Callable[[torch.Tensor], tuple], h: torch.Tensor, S: torch.Tensor, nalpha: int, nbeta: int,
        enuc: float, C0: Optional[tuple] = None, e_conv: float = 1e-10, d_conv: float = 1e-8, maxiter: int = 200,
        ndiis: int = 8, lindep: float = 1e-9, jk_batch: Optional[Callable[[list], list]] = None) -> dict:
    """Unrestricted SCF (the reference's ``UHF`` keyword of &SCF): separate
    alpha and beta orbitals, F_s = h + J[D_a + D_b] - K[D_s], two jk calls per
    iteration, one DIIS over both spin commutators.  jk_batch, when given,
    takes the list of occupied factors and returns their (J, K) in one call
    (MolGpu.cho_jk_batch: one pass over the Cholesky vectors for both spins,
    the two-density CHO_LK_SCF call of scf/choscf_drv.F90:433); jk is then
    not called.

    E = 1/2 tr((D_a + D_b) h) + 1/2 tr(D_a F_a) + 1/2 tr(D_b F_b) + enuc; its
    two-electron part equals 1/2 tr(D J[D]) - 1/4 (tr(D K[D]) + tr(DS K[DS]))
    with D = D_a + D_b and DS = D_a - D_b, the 2-PDM of PGet1 with the spin
    density, i.e. what ``mg_drvg1_x(h, D, DS, 1, 1, ...)`` differentiates.
    Returns dict(energy, C=(C_a, C_b), eps=(eps_a, eps_b), niter, converged,
    history)."""
    if maxiter < 1:
        raise ValueError("uhf: maxiter must be >= 1")
    dev, dt = h.device, torch.float64
    h = h.to(dev, dt)
    S = S.to(dev, dt)
    X = _orthogonaliser(S, lindep)
    if not (0 <= nbeta <= nalpha <= X.shape[1] and nalpha > 0):
        raise ValueError(f"uhf: {nalpha} alpha / {nbeta} beta electrons, {X.shape[1]} linearly independent functions")
    nocc = (nalpha, nbeta)

    def diag(F):
        eps, Ct = torch.linalg.eigh(X.T @ F @ X)
        return eps, X @ Ct

    if C0 is None:
        eps0, C = diag(h)
        Cs = [C, C]
        eps = [eps0, eps0]
    else:
        Cs = [c.to(dev, dt) for c in C0]
        eps = [None, None]
    fock_hist, err_hist, energies = [], [], []
    e_old = None
    converged = False
    for it in range(1, maxiter + 1):
        Ds, Ks = [], [torch.zeros_like(h), torch.zeros_like(h)]
        J = torch.zeros_like(h)
        occ = []
        for s in range(2):
            Co = Cs[s][:, :nocc[s]]
            Ds.append(Co @ Co.T)
            if nocc[s] > 0:
                occ.append((s, Co))
        res = jk_batch([Co for _, Co in occ]) if jk_batch is not None else [jk(Co) for _, Co in occ]
        for (s, _), (Js, Kk) in zip(occ, res):
            J = J + Js.to(dev, dt)
            Ks[s] = Kk.to(dev, dt)
        Fs = [h + J - Ks[s] for s in range(2)]
        E = float(0.5 * torch.sum((Ds[0] + Ds[1]) * h) + 0.5 * torch.sum(Ds[0] * Fs[0])
                  + 0.5 * torch.sum(Ds[1] * Fs[1])) + enuc
        energies.append(E)
        errs = [X.T @ (Fs[s] @ Ds[s] @ S - S @ Ds[s] @ Fs[s]) @ X for s in range(2)]
        emax = max(float(e.abs().max()) for e in errs)
        if e_old is not None and abs(E - e_old) < e_conv and emax < d_conv:
            converged = True
            for s in range(2):
                eps[s], Cs[s] = diag(Fs[s])
            break
        e_old = E
        fock_hist.append(Fs)
        err_hist.append(errs)
        del fock_hist[:-ndiis], err_hist[:-ndiis]
        n = len(fock_hist)
        if n > 1:
            Bm = torch.empty((n + 1, n + 1), dtype=dt, device=dev)
            for i in range(n):
                for j in range(n):
                    Bm[i, j] = torch.sum(err_hist[i][0] * err_hist[j][0]) + torch.sum(err_hist[i][1] * err_hist[j][1])
            Bm[n, :n] = -1.0
            Bm[:n, n] = -1.0
            Bm[n, n] = 0.0
            rhs = torch.zeros(n + 1, dtype=dt, device=dev)
            rhs[n] = -1.0
            try:
                c = torch.linalg.solve(Bm, rhs)[:n]
                Fs = [sum(ci * Fi[s] for ci, Fi in zip(c, fock_hist)) for s in range(2)]
            except RuntimeError:  # singular subspace: restart it from the newest Fock matrices
                del fock_hist[:-1], err_hist[:-1]
        for s in range(2):
            eps[s], Cs[s] = diag(Fs[s])
    return dict(energy=energies[-1], C=tuple(Cs), eps=tuple(eps), niter=len(energies), converged=converged,
                history=energies)
