"""Device paths against the reference's own regression tests (the checkfile
values of tests 020, 023, 065, 071 and 862, see tests/golden/): SCF energies
over the device ERIs and the device Cholesky J/K, and nuclear gradients with
the device Drvg1.  The oracle supplies the one-electron matrices and their
derivatives; the bars are the reference harness's own digits
(Tools/pymolcas/check_test.py:137-151), and each device part is also held to
the oracle's result for the same input."""
import numpy as np
import pytest
import torch

from conftest import exact_jk, full_eri_from_blocks
from oracle import oneint
from oracle import oracle as O
from openmolcas_b200 import scf
from openmolcas_b200.molgpu import MolGpu, unique_quartets

pytestmark = pytest.mark.gpu


def test_rhf_over_device_jk_scf065(scf065):
    mol, z, Cocc = scf065["mol"], scf065["z"], scf065["Cocc"]
    S, T, V = oneint.one_electron(mol)
    enuc = float(z["POTNUC"])
    nocc = Cocc.shape[1]
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-4)
    dev = torch.device("cuda", g.device)
    res = scf.rhf(lambda Cf: g.cho_jk(Cf, precision=MolGpu.PREC_FP64), torch.from_numpy(T + V).to(dev),
                  torch.from_numpy(S).to(dev), nocc, enuc)
    o = O.Oracle(mol)
    L = o.cholesky(thrcom=1e-4)["L"]

    def jk(Cf):
        J, K = o.cho_jk(L, Cf.numpy())
        return torch.from_numpy(J), torch.from_numpy(K)

    ref = scf.rhf(jk, torch.from_numpy(T + V), torch.from_numpy(S), nocc, enuc)
    print(f"065 SCF device: E = {res['energy']:.12f} ({res['niter']} it), oracle J/K {ref['energy']:.12f}")
    assert res["converged"] and ref["converged"]
    assert res["C"].is_cuda
    assert abs(res["energy"] - ref["energy"]) < 1e-8
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    assert np.isfinite(res["eps"].cpu().numpy()).all()


def test_reference_scf_device_eris_and_cholesky(refscf):
    """The reference's tests 071 (water, cc-pVTZ: d and f shells) and 004
    (water, ANO-S general contractions), conventional integrals, through the
    device: the SCF over every unique shell quartet from mg_eri_quartets, and
    over mg_cho_drv (ThrCom 1e-9) + mg_cho_jk FP64, both meet E_SCF to the
    checkfile's 8 digits; the Cholesky SCF equals the same loop over the
    oracle's vectors to 1e-8 (1e-10 relative: the FP64 J/K parity bar)."""
    mol, z, nocc = refscf["mol"], refscf["z"], refscf["nocc"]
    S, T, V = oneint.one_electron(mol)
    enuc = oneint.nuclear_repulsion(mol)
    bar = 10.0 ** -int(z["E_SCF_digits"])
    g = MolGpu(mol)
    o = O.Oracle(mol)
    q = unique_quartets(len(mol.shells))
    flat, off = g.eri_quartets(q)
    eri = full_eri_from_blocks(mol, q, flat.cpu().numpy(), off)
    assert np.abs(eri - o.eri_full()).max() < 1e-11
    h, Sm = torch.from_numpy(T + V), torch.from_numpy(S)
    r1 = scf.rhf(exact_jk(eri), h, Sm, nocc, enuc, e_conv=1e-12, d_conv=1e-10)
    assert r1["converged"] and abs(r1["energy"] - float(z["E_SCF"])) <= bar
    g.cho_drv(thrcom=1e-9)
    dev = torch.device("cuda", g.device)
    r2 = scf.rhf(lambda Cf: g.cho_jk(Cf, precision=MolGpu.PREC_FP64), h.to(dev), Sm.to(dev), nocc, enuc,
                 e_conv=1e-12, d_conv=1e-10)
    L = o.cholesky(thrcom=1e-9)["L"]

    def jk(Cf):
        J, K = o.cho_jk(L, Cf.numpy())
        return torch.from_numpy(J), torch.from_numpy(K)

    r3 = scf.rhf(jk, h, Sm, nocc, enuc, e_conv=1e-12, d_conv=1e-10)
    print(f"{mol.name} device: ERIs {r1['energy']:.12f}, Cholesky {r2['energy']:.12f}, E_SCF {float(z['E_SCF']):.12f}")
    assert r2["converged"] and abs(r2["energy"] - float(z["E_SCF"])) <= bar
    assert abs(r2["energy"] - r3["energy"]) < 1e-8


def test_grad862_device_eris_and_drvg1_against_reference(grad862):
    """The reference's test 862 (water, 6-31G, conventional integrals), first
    geometry, through the device: every unique shell quartet from
    mg_eri_quartets feeds the SCF (E_SCF to the checkfile's 8 digits), and
    mg_drvg1 gives the two-electron gradient, which with the oracle's
    one-electron and nuclear terms meets GRAD to its 6 digits; the device
    parts also equal the oracle's (1e-11 ERIs, 1e-9 relative gradient)."""
    mol, z, nocc = grad862["mol"], grad862["z"], grad862["nocc"]
    g = MolGpu(mol)
    o = O.Oracle(mol)
    q = unique_quartets(len(mol.shells))
    flat, off = g.eri_quartets(q)
    eri = full_eri_from_blocks(mol, q, flat.cpu().numpy(), off)
    assert np.abs(eri - o.eri_full()).max() < 1e-11
    S, T, V = oneint.one_electron(mol)
    res = scf.rhf(exact_jk(eri), torch.from_numpy(T + V), torch.from_numpy(S), nocc, oneint.nuclear_repulsion(mol),
                  e_conv=1e-12, d_conv=1e-10)
    assert res["converged"]
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    C, eps = res["C"].numpy(), res["eps"].numpy()
    Co = C[:, :nocc]
    D, W = 2.0 * Co @ Co.T, 2.0 * (Co * eps[:nocc]) @ Co.T
    g2 = g.drvg1(torch.from_numpy(D)).cpu().numpy()
    ref2 = o.grad(D)
    assert np.abs(g2 - ref2).max() < 1e-9 * max(1.0, np.abs(ref2).max())
    G = oneint.one_electron_gradient(mol, D, W) + g2 + oneint.nuclear_repulsion_gradient(mol)
    err = np.abs(G - z["GRAD"]).max()
    print(f"862 device: E = {res['energy']:.12f} (E_SCF {float(z['E_SCF']):.12f}), max |grad - GRAD| = {err:.1e}")
    assert err <= 10.0 ** -int(z["GRAD_digits"])


def test_symmetric_case_device_drvg1_with_d_shells_against_reference(symgrad):
    """The reference's tests 020 (CH4) and 023 (CH2O2), cc-pVDZ with d
    shells: the SCF over the device ERIs meets E_SCF (8 digits) and mg_drvg1
    gives the two-electron gradient, which with the oracle's one-electron and
    nuclear terms meets the checkfile's symmetry-reduced GRAD (6 digits)."""
    mol, z, nocc = symgrad["mol"], symgrad["z"], symgrad["nocc"]
    g = MolGpu(mol)
    o = O.Oracle(mol)
    q = unique_quartets(len(mol.shells))
    flat, off = g.eri_quartets(q)
    eri = full_eri_from_blocks(mol, q, flat.cpu().numpy(), off)
    S, T, V = oneint.one_electron(mol)
    res = scf.rhf(exact_jk(eri), torch.from_numpy(T + V), torch.from_numpy(S), nocc, oneint.nuclear_repulsion(mol),
                  e_conv=1e-12, d_conv=1e-10)
    assert res["converged"]
    assert abs(res["energy"] - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    C, eps = res["C"].numpy(), res["eps"].numpy()
    Co = C[:, :nocc]
    D, W = 2.0 * Co @ Co.T, 2.0 * (Co * eps[:nocc]) @ Co.T
    g2 = g.drvg1(torch.from_numpy(D)).cpu().numpy()
    ref2 = o.grad(D)
    assert np.abs(g2 - ref2).max() < 1e-9 * max(1.0, np.abs(ref2).max())
    G = oneint.one_electron_gradient(mol, D, W) + g2 + oneint.nuclear_repulsion_gradient(mol)
    err = np.abs(G[z["grad_atom"], z["grad_comp"]] - z["GRAD"]).max()
    print(f"{mol.name} device: max |grad - GRAD| = {err:.1e}")
    assert err <= 10.0 ** -int(z["GRAD_digits"])


def test_uhf_over_device_batched_jk_862(grad862):
    """Open-shell UHF (the water cation of test 862's basis and geometry, 5
    alpha and 4 beta electrons) over mg_cho_drv (ThrCom 1e-9) with both spins'
    J and K from one mg_cho_jk_batch call per iteration: equal to the same
    loop with two mg_cho_jk calls and to the loop over the oracle's vectors
    (1e-8 Eh), within 1e-6 Eh of UHF over exact integrals (the decomposition
    error), and the mixed-precision batch within 1e-8 Eh of the FP64 one."""
    mol = grad862["mol"]
    S, T, V = oneint.one_electron(mol)
    enuc = oneint.nuclear_repulsion(mol)
    h, Sm = torch.from_numpy(T + V), torch.from_numpy(S)
    o = O.Oracle(mol)
    kw = dict(e_conv=1e-12, d_conv=1e-10)
    r0 = scf.uhf(exact_jk(o.eri_full()), h, Sm, 5, 4, enuc, **kw)
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-9)
    dev = torch.device("cuda", g.device)
    hd, Sd = h.to(dev), Sm.to(dev)
    fp64 = MolGpu.PREC_FP64
    r1 = scf.uhf(None, hd, Sd, 5, 4, enuc, jk_batch=lambda Cs: g.cho_jk_batch(Cs, precision=fp64), **kw)
    r2 = scf.uhf(lambda Cf: g.cho_jk(Cf, precision=fp64), hd, Sd, 5, 4, enuc, **kw)
    r3 = scf.uhf(None, hd, Sd, 5, 4, enuc, jk_batch=lambda Cs: g.cho_jk_batch(Cs, precision=MolGpu.PREC_MIXED), **kw)
    L = o.cholesky(thrcom=1e-9)["L"]

    def jk(Cf):
        J, K = o.cho_jk(L, Cf.numpy())
        return torch.from_numpy(J), torch.from_numpy(K)

    r4 = scf.uhf(jk, h, Sm, 5, 4, enuc, **kw)
    print(f"UHF 862 cation: exact {r0['energy']:.12f}, device batch {r1['energy']:.12f}, two calls "
          f"{r2['energy']:.12f}, mixed batch {r3['energy']:.12f}, oracle vectors {r4['energy']:.12f}")
    assert all(r["converged"] for r in (r0, r1, r2, r3, r4))
    assert abs(r1["energy"] - r2["energy"]) < 1e-10
    assert abs(r1["energy"] - r4["energy"]) < 1e-8
    assert abs(r1["energy"] - r0["energy"]) < 1e-6
    assert abs(r3["energy"] - r1["energy"]) < 1e-8
