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
