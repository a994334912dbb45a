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


@pytest.fixture(scope="module")
def c2():
    mol = B.config_molecule("c2")  # 40 atoms, 600 functions, l <= 3, 1-12 primitives per shell
    g = MolGpu(mol)
    tm = g.schwarz()
    q = unique_quartets(len(mol.shells), tm, 1e-12)
    return mol, g, tm, q


def test_c2_cluster_sample_vs_oracle(c2):
    """A seeded sample of the 40-atom cluster's Schwarz-screened quartets
    against the oracle (every class of the uneven basis is drawn)."""
    mol, g, tm, q = c2
    rng = np.random.default_rng(4)
    sel = q[rng.choice(len(q), 300, replace=False)]
    assert _compare(mol, sel) <= 1.0


def test_c2_cluster_bra_ket_symmetry_and_schwarz(c2):
    """Size-independent properties on a 20 000-quartet slice of the full
    workload: (ij|kl) computed as (kl|ij) (the other class kernel, the other
    transfer centres) agrees element by element, and every integral obeys the
    Schwarz bound TMax(ij) TMax(kl)."""
    mol, g, tm, q = c2
    rng = np.random.default_rng(5)
    sel = q[rng.choice(len(q), 20000, replace=False)]
    swp = sel[:, [2, 3, 0, 1]].copy()
    a, offa = g.eri_quartets(sel)
    b, offb = g.eri_quartets(swp)
    a, b = a.cpu().numpy(), b.cpu().numpy()
    sh = mol.shells
    o = None
    nflag, worst = 0, 0.0
    for t, (i, j, k, l) in enumerate(sel):
        ni, nj, nk, nl = (sh[x].ncontr for x in (i, j, k, l))
        na, nb, nc, nd = (sh[x].ncomp for x in (i, j, k, l))
        A = a[offa[t]:offa[t + 1]].reshape(nd, nc, nb, na, nl, nk, nj, ni)
        Bq = b[offb[t]:offb[t + 1]].reshape(nb, na, nd, nc, nj, ni, nl, nk).transpose(2, 3, 0, 1, 6, 7, 4, 5)
        d = np.abs(A - Bq)
        assert np.abs(A).max() <= tm[i, j] * tm[k, l] * (1 + 1e-10) + 1e-12
        if (d <= 1e-11 + 1e-11 * np.abs(A)).all():
            continue
        # cancellation: hold the pair to twice the per-integral FP64 bar of the oracle's
        # cancellation-free magnitude
        o = o or O.Oracle(mol)
        S = o.eri_quartet_abs(int(i), int(j), int(k), int(l)).reshape(A.shape)
        worst = max(worst, float((d / (2 * O.eri_tolerance(S))).max()))
        nflag += 1
    print(f"bra-ket swap: {nflag} of {len(sel)} quartets beyond 1e-11 relative; worst vs 2x bar {worst:.3f}")
    assert worst <= 1.0
