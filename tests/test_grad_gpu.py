"""GPU two-electron gradient (adjoint Rys kernel) against the CPU oracle
(which is itself pinned to central finite differences in test_oracle.py).
Bar: 1e-8 Eh/bohr absolute (the north-star gradient bar is 1e-6)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mol", [
    B.small_molecule(3, seed=7),
    B.small_molecule(3, mix=[("4s3p2d1f_r", 2), ("2s1p", 1)], seed=21),
    B.make_molecule("c4like", 3, [("4s3p2d", 3)], 4),
])
def test_gradient_matches_oracle(mol):
    g = MolGpu(mol)
    o = O.Oracle(mol)
    Cm = B.density_factor(g.nbf, 6, 3)
    D = Cm @ Cm.T
    ref = o.grad(D)
    got = g.drvg1(torch.from_numpy(D)).cpu().numpy()
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(got - ref).max() < 1e-8 * scale, (got, ref)
    assert np.abs(got.sum(0)).max() < 1e-9 * scale


def test_gradient_repeatable_and_linear_in_scale():
    mol = B.small_molecule(3, seed=8)
    g = MolGpu(mol)
    Cm = B.density_factor(g.nbf, 5, 1)
    D = torch.from_numpy(Cm @ Cm.T)
    g1 = g.drvg1(D).cpu().numpy()
    g2 = g.drvg1(2.0 * D).cpu().numpy()  # quadratic in D
    assert np.abs(g2 - 4.0 * g1).max() < 1e-9 * max(1.0, np.abs(g2).max())
