"""SCF energies and nuclear gradients against the reference's regression
tests (the checkfile values of tests 862, 020, 023, 019, 021, 049 and 094; the
energy-only cases are in test_scf.py), with the oracle's ERIs, one-electron
matrices and Drvg1 restatement, and the SCF loop of openmolcas_b200/scf.py.
The bars are the reference harness's own (E_SCF 8 digits, GRAD 6 digits;
Tools/pymolcas/check_test.py:137-151)."""
import numpy as np
import torch

from conftest import exact_jk, full_eri_from_blocks
from oracle import oneint
from oracle import oracle as O
from openmolcas_b200 import scf
from openmolcas_b200.molgpu import unique_quartets


def _scf(mol, eri, nocc):
    S, T, V = oneint.one_electron(mol)
    res = scf.rhf(exact_jk(eri), torch.from_numpy(T + V), torch.from_numpy(S), nocc, oneint.nuclear_repulsion(mol),
                  e_conv=1e-12, d_conv=1e-10)
    C, eps = res["C"].numpy(), res["eps"].numpy()
    Co = C[:, :nocc]
    return res, 2.0 * Co @ Co.T, 2.0 * (Co * eps[:nocc]) @ Co.T


def test_full_eri_from_blocks_matches_oracle(grad862):
    mol = grad862["mol"]
    o = O.Oracle(mol)
    q = unique_quartets(len(mol.shells))
    blocks = [o.eri_quartet(*map(int, t)) for t in q]
    off = np.concatenate([[0], np.cumsum([b.size for b in blocks])])
    eri = full_eri_from_blocks(mol, q, np.concatenate(blocks), off)
    assert np.abs(eri - o.eri_full()).max() < 1e-14


def test_grad862_energy_and_gradient_oracle(grad862):
    mol, z, nocc = grad862["mol"], grad862["z"], grad862["nocc"]
    o = O.Oracle(mol)
    res, D, W = _scf(mol, o.eri_full(), nocc)
    e_ref = float(z["E_SCF"])
    print(f"862: E = {res['energy']:.12f}  E_SCF = {e_ref:.12f}  dE = {res['energy'] - e_ref:.1e}")
    assert res["converged"]
    assert abs(res["energy"] - e_ref) <= 10.0 ** -int(z["E_SCF_digits"])
    G = oneint.one_electron_gradient(mol, D, W) + o.grad(D) + oneint.nuclear_repulsion_gradient(mol)
    err = np.abs(G - z["GRAD"]).max()
    print(f"862: max |grad - GRAD| = {err:.1e}")
    assert err <= 10.0 ** -int(z["GRAD_digits"])
    assert np.abs(G.sum(0)).max() < 1e-10


def test_one_electron_gradient_vs_central_fd(grad862):
    """d/dR [tr(D h(R)) - tr(W S(R))] at fixed D, W, by central differences."""
    mol = grad862["mol"]
    rng = np.random.default_rng(0)
    n = mol.nbf
    A = rng.standard_normal((n, n))
    D = A + A.T
    B_ = rng.standard_normal((n, n))
    W = B_ + B_.T
    G = oneint.one_electron_gradient(mol, D, W)
    h = 1e-5
    for at, ax in [(0, 2), (1, 0), (2, 1)]:
        def e1(m):
            S, T, V = oneint.one_electron(m)
            return np.sum(D * (T + V)) - np.sum(W * S)
        fd = (e1(mol.moved(at, ax, h)) - e1(mol.moved(at, ax, -h))) / (2 * h)
        assert abs(fd - G[at, ax]) < 1e-6 * max(1.0, abs(fd))


def test_symmetric_case_energy_and_symmetry_unique_gradient(symgrad_all):
    """The reference's tests 020 (CH4) and 023 (CH2O2) in cc-pVDZ (d shells on
    the heavy atoms), 019 (C4H8) and 021 (benzene) in STO-3G, point-group
    symmetry in the reference and all atoms here: E_SCF to its 8 digits and
    the GRAD entries (symmetry-allowed components of the unique centres) to
    their 6 digits."""
    mol, z, nocc = symgrad_all["mol"], symgrad_all["z"], symgrad_all["nocc"]
    assert abs(oneint.nuclear_repulsion(mol) - float(z["POTNUC"])) <= 10.0 ** -int(z["POTNUC_digits"])
    o = O.Oracle(mol)
    res, D, W = _scf(mol, o.eri_full(), nocc)
    assert res["converged"]
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    G = oneint.one_electron_gradient(mol, D, W) + o.grad(D) + oneint.nuclear_repulsion_gradient(mol)
    g = G[z["grad_atom"], z["grad_comp"]]
    err = np.abs(g - z["GRAD"]).max()
    print(f"{mol.name}: E - E_SCF = {res['energy'] - float(z['E_SCF']):.1e}, max |grad - GRAD| = {err:.1e}")
    assert err <= 10.0 ** -int(z["GRAD_digits"])


def test_scf049_ch2o2_energy():
    """The reference's test 049 (CH2O2 transition-state search, cc-pVDZ, Cs):
    E_SCF of the first geometry to its 8 digits.  Its GRAD is not asserted:
    that run used Alaska's default screening of gradient contributions
    (CutGrd = 1e-7, alaska/inputg.F90:109-112), and the unscreened gradient
    here differs from it by up to 1.3e-6 Eh/bohr, above the harness's 1e-6
    (test 862, run with CUTOFF=1.0D-8, agrees to 1.7e-7)."""
    from conftest import _symgrad_case
    c = _symgrad_case("grad049_ch2o2_ccpvdz")
    mol, z, nocc = c["mol"], c["z"], c["nocc"]
    res, _, _ = _scf(mol, O.Oracle(mol).eri_full(), nocc)
    assert res["converged"]
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])


def test_grad094_hcn_sto3g_energy_and_gradient():
    """The reference's test 094 (HCN/CNH, STO-3G, no symmetry; &SCF then
    &SLAPAF, which has Alaska compute the SCF gradient): E_SCF to its 8 digits
    and the first GRAD to its 6 digits."""
    from conftest import _symgrad_case
    c = _symgrad_case("scf094_hcn_sto3g")
    mol, z, nocc = c["mol"], c["z"], c["nocc"]
    o = O.Oracle(mol)
    res, D, W = _scf(mol, o.eri_full(), nocc)
    assert res["converged"]
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    G = oneint.one_electron_gradient(mol, D, W) + o.grad(D) + oneint.nuclear_repulsion_gradient(mol)
    assert np.abs(G - z["GRAD"]).max() <= 10.0 ** -int(z["GRAD_digits"])
