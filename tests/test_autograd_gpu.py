"""The differentiable J/K energy: backward (the gradient kernel and
dE/dC = 2(J - K/2)C) against central finite differences of the forward
(h = 1e-4 bohr, bar 1e-6 Eh/bohr), and mg_rys_roots (the device
table evaluation) against the reference's own Rys table values."""
import os

import numpy as np
import pytest
import torch

from openmolcas_b200 import basis as B

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.gpu
def test_jk_energy_backward_matches_finite_differences():
    from openmolcas_b200.autograd import jk_energy
    m = B.small_molecule(3, mix=[("3s2p1d", 3)], seed=5)
    Cm = torch.from_numpy(B.density_factor(m.nbf, 4, 9))
    R = torch.tensor(m.coords, dtype=torch.float64, requires_grad=True)
    Cp = Cm.clone().requires_grad_(True)
    kw = dict(thrcom=1e-12)
    E = jk_energy(R, Cp, m, **kw)
    E.backward()
    gR, gC = R.grad.clone(), Cp.grad.clone()
    h = 1e-4
    worst = 0.0
    for atom, axis in [(0, 0), (1, 2), (2, 1)]:
        Rp, Rm = R.detach().clone(), R.detach().clone()
        Rp[atom, axis] += h
        Rm[atom, axis] -= h
        fd = (jk_energy(Rp, Cm, m, **kw) - jk_energy(Rm, Cm, m, **kw)).item() / (2 * h)
        worst = max(worst, abs(fd - gR[atom, axis].item()))
    print(f"max |dE/dR - FD| = {worst:.2e} (scale {gR.abs().max().item():.2f})")
    assert worst < 1e-6
    assert abs(gR.sum(0)).max().item() < 1e-9  # translational invariance
    for (a, k) in [(0, 0), (5, 2), (11, 3)]:
        Cp_, Cm_ = Cm.clone(), Cm.clone()
        Cp_[a, k] += h
        Cm_[a, k] -= h
        fd = (jk_energy(R.detach(), Cp_, m, **kw) - jk_energy(R.detach(), Cm_, m, **kw)).item() / (2 * h)
        assert abs(fd - gC[a, k].item()) < 1e-6 * max(1.0, abs(fd))


@pytest.mark.gpu
def test_device_rys_table_vs_reference_golden():
    from openmolcas_b200.molgpu import MolGpu
    g = MolGpu(B.small_molecule(2))
    gold = np.load(os.path.join(GOLD, "rys_ref.npz"))
    for n in range(1, 10):
        T = gold[f"T{n}"]
        x, w = g.rys_roots(n, T)
        acc = max(gold["acc"][n - 1], 2e-15)
        rx = np.abs(x - gold[f"x{n}"]) / np.abs(gold[f"x{n}"])
        rw = np.abs(w - gold[f"w{n}"]) / np.abs(gold[f"w{n}"]).max(axis=1, keepdims=True)
        assert rx.max() < 10 * acc, (n, rx.max())
        assert rw.max() < 10 * acc, (n, rw.max())
    # Sigma w = F0(T), asymptotic branch included
    T = np.array([0.0, 0.7, 30.0, 150.0])
    x, w = g.rys_roots(5, T)
    import math
    f0 = np.array([1.0 if t == 0 else 0.5 * math.sqrt(math.pi / t) * math.erf(math.sqrt(t)) for t in T])
    assert np.allclose(w.sum(1), f0, rtol=1e-13)
