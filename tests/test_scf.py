"""SCF caller loop (openmolcas_b200/scf.py) on the CPU with the oracle's
Cholesky J/K, on the reference's test 065 (CO, cc-pVDZ, ThrCom 1e-4).

From a core-Hamiltonian guess the iteration reaches the energy of the
orbitals embedded in test 065 (which are converged for these vectors to
1e-8 Eh), lies at or below it (variational), and meets E_SCF within the
reference harness's tolerance for it (10^-4)."""
import math

import numpy as np
import torch

from conftest import rhf_energy
from oracle import oneint
from oracle import oracle as O
from openmolcas_b200 import scf


def test_rhf_converges_to_scf065_energy(scf065):
    mol, z, Cocc = scf065["mol"], scf065["z"], scf065["Cocc"]
    S, T, V = oneint.one_electron(mol)
    o = O.Oracle(mol)
    L = o.cholesky(thrcom=1e-4)["L"]

    def jk(Cf):
        J, K = o.cho_jk(L, Cf.numpy())
        return torch.from_numpy(J), torch.from_numpy(K)

    enuc = float(z["POTNUC"])
    res = scf.rhf(jk, torch.from_numpy(T + V), torch.from_numpy(S), Cocc.shape[1], enuc)
    J, K = o.cho_jk(L, math.sqrt(2.0) * Cocc)
    e_frozen = rhf_energy(T + V, J, K, 2.0 * Cocc @ Cocc.T, enuc)
    print(f"SCF: E = {res['energy']:.12f} in {res['niter']} iterations; embedded orbitals {e_frozen:.12f}")
    assert res["converged"]
    assert res["energy"] <= e_frozen + 1e-10
    assert abs(res["energy"] - e_frozen) < 1e-7
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    # the occupied space is the embedded one (to ~sqrt of the 1e-8 Eh gap)
    C = res["C"].numpy()[:, : Cocc.shape[1]]
    P1, P0 = C @ C.T, Cocc @ Cocc.T
    assert np.abs(P1 - P0).max() < 1e-3
    # starting from the embedded orbitals the energy only drops by the last 1e-8
    res2 = scf.rhf(jk, torch.from_numpy(T + V), torch.from_numpy(S), Cocc.shape[1], enuc,
                   C0=torch.from_numpy(Cocc))
    assert abs(res2["history"][0] - e_frozen) < 1e-12
    assert abs(res2["energy"] - res["energy"]) < 1e-9


def _rhf_ref(mol, nocc, jk, z):
    """SCF from a core guess, or from the orbitals the reference test embeds
    (``orbitals`` in the fixture), as that test's &SCF starts."""
    S, T, V = oneint.one_electron(mol)
    C0 = torch.from_numpy(z["orbitals"].T.copy()) if "orbitals" in z else None
    return scf.rhf(jk, torch.from_numpy(T + V), torch.from_numpy(S), nocc, oneint.nuclear_repulsion(mol),
                   C0=C0, e_conv=1e-12, d_conv=1e-10)


def test_reference_scf_energy_exact_and_cholesky(refscf_all):
    """The reference's tests 071 (water, cc-pVTZ with d and f shells), 004
    (water, ANO-S general contractions) and 007 (CH2, inline basis),
    conventional integrals: the SCF over
    the oracle's exact ERIs meets E_SCF (checked to 8 digits by the reference
    harness) and POTNUC (12 digits); over Cholesky vectors at ThrCom 1e-9 it
    stays within the same 1e-8."""
    from conftest import exact_jk
    mol, z, nocc = refscf_all["mol"], refscf_all["z"], refscf_all["nocc"]
    assert abs(oneint.nuclear_repulsion(mol) - float(z["POTNUC"])) <= 10.0 ** -int(z["POTNUC_digits"])
    o = O.Oracle(mol)
    bar = 10.0 ** -int(z["E_SCF_digits"])
    res = _rhf_ref(mol, nocc, exact_jk(o.eri_full()), z)
    print(f"{mol.name}: E = {res['energy']:.12f}  E_SCF = {float(z['E_SCF']):.12f}")
    assert res["converged"] and abs(res["energy"] - float(z["E_SCF"])) <= bar
    L = o.cholesky(thrcom=1e-9)["L"]

    def jk(Cf):
        J, K = o.cho_jk(L, Cf.numpy())
        return torch.from_numpy(J), torch.from_numpy(K)

    rc = _rhf_ref(mol, nocc, jk, z)
    assert rc["converged"] and abs(rc["energy"] - float(z["E_SCF"])) <= bar


def test_rhf_rejects_bad_arguments():
    import pytest
    h = torch.eye(3, dtype=torch.float64)
    S = torch.eye(3, dtype=torch.float64)

    def jk(Cf):
        return torch.zeros(3, 3, dtype=torch.float64), torch.zeros(3, 3, dtype=torch.float64)

    with pytest.raises(ValueError):
        scf.rhf(jk, h, S, 4, 0.0)
    with pytest.raises(ValueError):
        scf.rhf(jk, h, S, 1, 0.0, maxiter=0)
    res = scf.rhf(jk, h, S, 2, 1.0)  # no two-electron term: E = 2 * 2 * 1 + 1
    assert res["converged"] and abs(res["energy"] - 5.0) < 1e-12


def _uhf(mol, na, nb):
    from conftest import exact_jk
    S, T, V = oneint.one_electron(mol)
    o = O.Oracle(mol)
    return scf.uhf(exact_jk(o.eri_full()), torch.from_numpy(T + V), torch.from_numpy(S), na, nb,
                   oneint.nuclear_repulsion(mol), e_conv=1e-12, d_conv=1e-10), o


def test_uhf_closed_shell_limit_is_scf862(grad862):
    """With equal alpha and beta occupations UHF is RHF: test 862's E_SCF."""
    mol, z = grad862["mol"], grad862["z"]
    res, _ = _uhf(mol, 5, 5)
    assert res["converged"] and abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])


def test_uhf_gradient_with_spin_density_vs_central_fd(grad862):
    """H2O+ doublet (5 alpha, 4 beta) in 6-31G: the nuclear gradient from
    the spin-density 2-PDM (oracle Drvg1 with DS = D_a - D_b, the input of
    mg_drvg1_x), the one-electron terms with W = sum_s C_s eps_s C_s^T and
    the nuclear repulsion equals central differences of converged UHF
    energies."""
    mol = grad862["mol"]
    res, o = _uhf(mol, 5, 4)
    assert res["converged"]
    (Ca, Cb), (ea, eb) = [c.numpy() for c in res["C"]], [e.numpy() for e in res["eps"]]
    Da, Db = Ca[:, :5] @ Ca[:, :5].T, Cb[:, :4] @ Cb[:, :4].T
    W = (Ca[:, :5] * ea[:5]) @ Ca[:, :5].T + (Cb[:, :4] * eb[:4]) @ Cb[:, :4].T
    G = (oneint.one_electron_gradient(mol, Da + Db, W) + o.grad(Da + Db, DS=Da - Db)
         + oneint.nuclear_repulsion_gradient(mol))
    assert np.abs(G.sum(0)).max() < 1e-10
    h = 1e-4
    for at, ax in [(0, 2), (1, 0), (2, 2)]:
        ep = _uhf(mol.moved(at, ax, h), 5, 4)[0]["energy"]
        em = _uhf(mol.moved(at, ax, -h), 5, 4)[0]["energy"]
        assert abs((ep - em) / (2 * h) - G[at, ax]) < 1e-7
