"""SCF caller loop over the device Cholesky J/K (mg_cho_drv + mg_cho_jk FP64),
the dense algebra on the same GPU, for the reference's test 065 (CO,
cc-pVDZ): converges to the energy the same loop reaches with the oracle's
J/K (same pivots, vectors equal to rounding) and meets E_SCF within the
reference harness's tolerance for it (10^-4)."""
import numpy as np
import pytest
import torch

from oracle import oneint
from oracle import oracle as O
from openmolcas_b200 import scf
from openmolcas_b200.molgpu import MolGpu

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


def test_scf071_ccpvtz_device_eris_and_cholesky(scf071):
    """The reference's test 071 (water, cc-pVTZ: d and f shells, conventional
    integrals) through the device: the SCF over every unique shell quartet
    from mg_eri_quartets, and over mg_cho_drv (ThrCom 1e-9) + mg_cho_jk FP64,
    both meet E_SCF to the checkfile's 8 digits; the Cholesky SCF equals the
    same loop over the oracle's vectors to 1e-9."""
    from conftest import exact_jk, full_eri_from_blocks
    from openmolcas_b200.molgpu import unique_quartets

    mol, z, nocc = scf071["mol"], scf071["z"], scf071["nocc"]
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
    print(f"071 device: ERIs {r1['energy']:.12f}, Cholesky {r2['energy']:.12f}, E_SCF {float(z['E_SCF']):.12f}")
    assert r2["converged"] and abs(r2["energy"] - float(z["E_SCF"])) <= bar
    assert abs(r2["energy"] - r3["energy"]) < 1e-9
