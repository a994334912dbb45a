"""The oracle's instrumented build (oracle/_build/liboracle_count.so): the
restated ERI and gradient loops tally the FP64 operations they execute, per
stage.  This is the independent count that the kernels' own work models
(mg_eri_work, mg_drvg1_flops) are checked against in test_flops_gpu.py.
CPU only: a closed-form case, agreement with the default build, additivity
and a tally that does not depend on the OpenMP schedule."""
import numpy as np
import pytest

from oracle import oracle as O
from openmolcas_b200 import basis as B

ZERO = dict.fromkeys(O.FLOP_STAGES, 0.0)


def _two_s_atoms(dist):
    """One s shell of one primitive on each of two atoms `dist` bohr apart."""
    return B.molecule_from_arrays("ss", [[0.0, 0.0, 0.0], [0.0, 0.0, dist]], [1.0, 1.0], [0, 1], [0, 0], [1, 1],
                                  [1, 1], [0.5, 0.5], [1.0, 1.0])


def test_default_build_has_no_tally():
    with pytest.raises(RuntimeError):
        O.Oracle(_two_s_atoms(2.0)).flops()


def test_ssss_closed_form_count():
    """(s_A s_A | s_B s_B), one primitive per shell, 100 bohr apart: T is far
    above the table range, so every stage has a closed form -- set-up 16
    (zeta + eta, 1/(zeta + eta), rho, |PQ|^2, T, prefactor with its square
    root), asymptotic roots 2 + 2 n = 4, 2D coefficients 4 + 10 + 3 x 10 = 44,
    RysEF 3 + 1, contraction 1 + 2 + 2, HRR/spherical 2 + 2."""
    o = O.Oracle(_two_s_atoms(100.0), counting=True)
    o.flops(reset=True)
    o.eri_quartet(0, 0, 1, 1)
    want = dict(ZERO, prim=16, roots=4, rys2d=44, rysef=4, contract=5, hrr=4)
    assert o.flops() == want


def test_counting_build_same_integrals_and_additive():
    mol = B.small_molecule(3, seed=7)
    od, oc = O.Oracle(mol), O.Oracle(mol, counting=True)
    quartets = [(3, 1, 2, 0), (4, 4, 1, 0), (5, 2, 5, 3)]
    per = []
    for q in quartets:
        oc.flops(reset=True)
        a, b = od.eri_quartet(*q), oc.eri_quartet(*q)
        assert np.array_equal(a, b)  # the tally does not touch the arithmetic
        per.append(oc.flops())
        assert per[-1]["rysef"] > 0 and per[-1]["transfer"] == 0
    oc.flops(reset=True)
    for q in quartets:
        oc.eri_quartet(*q)
    total = oc.flops()
    for s in O.FLOP_STAGES:
        assert total[s] == sum(p[s] for p in per)


def test_gradient_tally_independent_of_schedule():
    """The gradient runs its quartets on OpenMP threads; each thread's tally is
    merged at the end of every quartet, so two runs count the same."""
    mol = B.make_molecule("c4like", 3, [("4s3p2d", 3)], 4)
    o = O.Oracle(mol, counting=True)
    Cm = B.density_factor(o.nbf, 6, 3)
    D = Cm @ Cm.T
    o.schwarz()  # the screening's own ERIs are not part of the gradient's count
    counts = []
    for _ in range(2):
        o.flops(reset=True)
        g = o.grad(D, cutint=1e-12)
        counts.append(o.flops())
    assert counts[0] == counts[1]
    c = counts[0]
    assert c["rysef"] == 0 and c["contract"] == 0 and c["hrr"] == 0
    assert min(c["assg1"], c["transfer"], c["pdm"], c["rys2d"]) > 0
    gd = O.Oracle(mol).grad(D, cutint=1e-12)
    assert np.allclose(g, gd, rtol=0, atol=1e-12 * np.abs(gd).max())
