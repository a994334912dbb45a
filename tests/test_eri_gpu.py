"""GPU parity of the FP64 Rys ERI kernels against the CPU oracle.

Bar per integral: |ERI_gpu - ERI_oracle| <= 1e-11 + 1e-13 * S, S the
cancellation-free magnitude of the integral (oracle with |coefficients|).
For well-conditioned contractions S ~ |ERI| and this is the 1e-11 absolute
bar; random-sign general contractions over exponents spanning four decades
cancel by up to ~1e7, where no FP64 summation order can hold 1e-11 (the
oracle against itself with permuted primitives differs by up to 9e-15*S)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, unique_quartets

pytestmark = pytest.mark.gpu


def _compare(mol, quartets):
    """Returns the largest error / tolerance ratio (must be <= 1)."""
    g = MolGpu(mol)
    o = O.Oracle(mol)
    out, off = g.eri_quartets(quartets)
    got = out.cpu().numpy()
    worst, nbig, ntot, wabs = 0.0, 0, 0, 0.0
    for t, (i, j, k, l) in enumerate(quartets):
        ref = o.eri_quartet(int(i), int(j), int(k), int(l))
        S = o.eri_quartet_abs(int(i), int(j), int(k), int(l))
        blk = got[off[t]:off[t + 1]]
        assert blk.size == ref.size
        d = np.abs(blk - ref)
        worst = max(worst, float((d / O.eri_tolerance(S)).max()))
        wabs = max(wabs, float(d.max()))
        nbig += int((d > O.ERI_ABS_TOL).sum())
        ntot += d.size
    print(f"max |d| {wabs:.2e}; {nbig}/{ntot} integrals above 1e-11 (all within 1e-11+1e-13*S)")
    return worst


def test_eri_all_classes_small_molecule():
    mol = B.small_molecule(3, seed=5)  # s,p,d,f shells, 1-12 primitives, general contraction
    q = unique_quartets(len(mol.shells))
    assert _compare(mol, q) <= 1.0


def test_eri_noncanonical_pair_order_and_repeats():
    mol = B.small_molecule(3, seed=9)
    ns = len(mol.shells)
    rng = np.random.default_rng(0)
    q = []
    for _ in range(200):
        i, j = sorted(rng.integers(0, ns, 2))[::-1]
        k, l = sorted(rng.integers(0, ns, 2))[::-1]
        q.append((i, j, k, l))  # (ij) < (kl) allowed
    assert _compare(mol, np.array(q, np.int32)) <= 1.0


def test_eri_six_atom_cluster_sample():
    mol = B.config_molecule("c1")
    q = unique_quartets(len(mol.shells))
    rng = np.random.default_rng(1)
    sel = q[rng.choice(len(q), 600, replace=False)]
    assert _compare(mol, sel) <= 1.0


def test_schwarz_matches_oracle():
    mol = B.small_molecule(4, mix=[("4s3p2d1f_r", 2), ("2s1p", 2)], seed=3)
    g = MolGpu(mol)
    o = O.Oracle(mol)
    tg, to = g.schwarz() ** 2, o.schwarz() ** 2  # max |(ab|ab)| per shell pair
    ns = len(mol.shells)
    for i in range(ns):
        for j in range(i + 1):
            S = o.eri_quartet_abs(i, j, i, j).max()
            assert abs(tg[i, j] - to[i, j]) <= O.eri_tolerance(S), (i, j, tg[i, j], to[i, j], S)


def test_eri_rejects_noncanonical_shell_pair():
    mol = B.small_molecule(2, seed=1)
    g = MolGpu(mol)
    with pytest.raises(RuntimeError):
        g.eri_quartets(np.array([[0, 1, 0, 0]], np.int32))
