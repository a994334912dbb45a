"""CPU tests of the oracle (test infrastructure) and of the host-side basis code.

They pin the oracle against: the reference's own Rys table (golden vectors
from data/rysrw.ascii), exact mpmath quadrature, the closed-form (ss|ss),
8-fold permutational symmetry, Cholesky reconstruction (the Cho_X_CheckDiag /
CD_Tester criterion), J/K from exact integrals and central finite
differences of the energy."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from openmolcas_b200 import basis as B

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_rys_table_vs_reference_golden():
    g = np.load(os.path.join(GOLD, "rys_ref.npz"))
    for n in range(1, 10):
        T = g[f"T{n}"]
        x, w = O.rys_rw(n, T)
        acc = max(g["acc"][n - 1], 2e-15)
        rx = np.abs(x - g[f"x{n}"]) / np.abs(g[f"x{n}"])
        rw = np.abs(w - g[f"w{n}"]) / np.abs(g[f"w{n}"]).max(axis=1, keepdims=True)
        assert rx.max() < 10 * acc, (n, rx.max())
        assert rw.max() < 10 * acc, (n, rw.max())


def test_rys_table_vs_mpmath():
    from openmolcas_b200.rys import gen_rys_tables as G
    from mpmath import mp
    mp.dps = 50
    rng = np.random.default_rng(3)
    for n in (1, 3, 5, 7):
        for T in list(rng.uniform(0, 100, 6)) + [0.0, 1e-6]:
            xe, we = G.rys_exact(n, T) if T < 90 else G.rys_asym(n, T)
            x, w = O.rys_rw(n, np.array([T]))
            assert np.allclose(x[0], [float(v) for v in xe], rtol=5e-15, atol=0)
            assert np.allclose(w[0], [float(v) for v in we], rtol=0, atol=5e-15 * float(max(we)))


def test_rys_weights_sum_to_boys_f0():
    T = np.array([0.0, 0.3, 2.0, 15.0, 45.0, 120.0])
    for n in range(1, 10):
        x, w = O.rys_rw(n, T)
        f0 = np.array([1.0 if t == 0 else 0.5 * math.sqrt(math.pi / t) * math.erf(math.sqrt(t)) for t in T])
        assert np.allclose(w.sum(1), f0, rtol=1e-13)


def test_spherical_d_and_p_conventions():
    S1 = O.sph_matrix(1)
    assert np.allclose(S1, np.eye(3))  # p stays Cartesian
    S2 = O.sph_matrix(2)  # columns m=-2..2 over xx,xy,xz,yy,yz,zz
    assert np.allclose(S2[:, 0], [0, 1, 0, 0, 0, 0])
    assert np.allclose(S2[:, 2] / S2[5, 2], [-0.5, 0, 0, -0.5, 0, 1])
    assert np.allclose(S2[:, 4], [0.5, 0, 0, -0.5, 0, 0])


def test_nrmlz_unit_self_overlap():
    rng = np.random.default_rng(0)
    for l in range(4):
        e = 0.08 * 3.0 ** np.arange(5)
        c = B.nrmlz(e, rng.standard_normal((5, 2)), l)
        # self-overlap of the x^l component: (2l-1)!! (Nrmlz leaves the double
        # factorial to the spherical normalisation NrmSph)
        df = float(np.prod(np.arange(2 * l - 1, 0, -2))) if l > 0 else 1.0
        S = df * math.pi ** 1.5 / (2.0 ** l * (e[:, None] + e[None, :]) ** (l + 1.5))
        ov = np.einsum("pi,pq,qi->i", c, S, c)
        assert np.allclose(ov, df, rtol=1e-12)


def _prim_mol(alphas, centers):
    shells = []
    for i, (a, c) in enumerate(zip(alphas, centers)):
        e = np.array([a])
        shells.append(B.Shell(i, 0, np.array(c, float), e, B.nrmlz(e, np.ones((1, 1)), 0)))
    return B.Molecule("p", np.array(centers, float), np.ones(len(alphas)), shells, 0)


def test_ssss_closed_form():
    al = [0.5, 1.3, 0.7, 2.1]
    cs = [[0, 0, 0], [1, 0.2, 0], [0, 1.5, 0.3], [0.4, 0.1, 2.0]]
    o = O.Oracle(_prim_mol(al, cs))
    v = o.eri_quartet(0, 1, 2, 3)[0]
    a, b, c, d = al
    A, Bc, Cc, D = [np.array(x, float) for x in cs]
    p, q = a + b, c + d
    P, Q = (a * A + b * Bc) / p, (c * Cc + d * D) / q
    T = p * q / (p + q) * np.sum((P - Q) ** 2)
    F0 = 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
    N = lambda x: (2 * x / math.pi) ** 0.75
    ref = (N(a) * N(b) * N(c) * N(d) * 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q))
           * math.exp(-a * b / p * np.sum((A - Bc) ** 2) - c * d / q * np.sum((Cc - D) ** 2)) * F0)
    assert abs(v - ref) < 1e-15


@pytest.fixture(scope="module")
def small():
    mol = B.small_molecule(3, seed=5)
    o = O.Oracle(mol)
    return mol, o, o.eri_full()


def test_eri_permutational_symmetry(small):
    mol, o, eri = small
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1), (3, 2, 1, 0)]:
        assert np.abs(eri - eri.transpose(*perm)).max() < 1e-12


def test_eri_blocks_all_orders_consistent(small):
    mol, o, eri = small
    off = np.cumsum([0] + [s.nbf for s in mol.shells])
    rng = np.random.default_rng(1)
    ns = len(mol.shells)
    for _ in range(40):
        i, j, k, l = rng.integers(0, ns, 4)
        blk = o.eri_quartet(i, j, k, l).reshape(o.quartet_shape(i, j, k, l))
        S = [mol.shells[x] for x in (i, j, k, l)]
        sub = eri[off[i]:off[i + 1], off[j]:off[j + 1], off[k]:off[k + 1], off[l]:off[l + 1]]
        # full AO index = off + m*nc + c  -> reshape to [m][c]
        sub = sub.reshape(S[0].ncomp, S[0].ncontr, S[1].ncomp, S[1].ncontr, S[2].ncomp, S[2].ncontr,
                          S[3].ncomp, S[3].ncontr)
        ref = sub.transpose(6, 4, 2, 0, 7, 5, 3, 1).reshape(blk.shape[:4] + (-1,))
        # blk[..., ijkl] with i fastest  <->  ref[..., (c_l, c_k, c_j, c_i)] C-order -> flip
        nc = [s.ncontr for s in S]
        got = blk.reshape(blk.shape[:4] + (nc[3], nc[2], nc[1], nc[0]))
        assert np.abs(got.reshape(ref.shape) - ref).max() < 1e-12


def test_eri_matrix_positive_semidefinite(small):
    mol, o, eri = small
    n = o.nbf
    ev = np.linalg.eigvalsh(eri.reshape(n * n, n * n))
    assert ev.min() > -1e-12 * ev.max()


def test_cholesky_reconstruction_and_pivots(small):
    mol, o, eri = small
    res = o.cholesky(thrcom=1e-6)
    a, b, sp = o.rs_list()
    L = res["L"]
    exact = eri[a[:, None], b[:, None], a[None, :], b[None, :]]
    rec = L @ L.T
    assert np.abs(rec - exact).max() <= 1e-6 * 1.0001
    assert np.all(np.diag(exact) - np.diag(rec) > -1e-12)
    assert len(set(res["piv"].tolist())) == res["M"]


def test_cho_jk_matches_exact_within_cd_error(small):
    mol, o, eri = small
    res = o.cholesky(thrcom=1e-8)
    Cm = B.density_factor(o.nbf, 5, 2)
    D = Cm @ Cm.T
    J, K = o.cho_jk(res["L"], Cm)
    E, Je, Ke = O.energy_from_full(eri, D)
    scale = np.abs(D).sum()
    assert np.abs(J - Je).max() < 1e-8 * scale
    assert np.abs(K - Ke).max() < 1e-8 * scale


def test_cho_jk_blas_equals_loop_restatement(small):
    """The BLAS-driven J/K (the timed CPU baseline) and the oracle's loop
    restatement of CHO_LK_SCF agree to rounding."""
    mol, o, eri = small
    res = o.cholesky(thrcom=1e-8)
    Cm = B.density_factor(o.nbf, 7, 3)
    J, K = o.cho_jk(res["L"], Cm)
    a, b, _ = o.rs_list()
    Jb, Kb = O.cho_jk_blas(a, b, o.nbf, res["L"], Cm, batch=5)
    assert np.abs(Jb - J).max() < 1e-12 * np.abs(J).max()
    assert np.abs(Kb - K).max() < 1e-12 * np.abs(K).max()


def test_gradient_vs_central_fd():
    mol = B.small_molecule(3, seed=7)
    o = O.Oracle(mol)
    Cm = B.density_factor(o.nbf, 4, 3)
    D = Cm @ Cm.T
    g = o.grad(D)
    assert np.abs(g.sum(0)).max() < 1e-10  # translational invariance
    h = 1e-4
    for at, ax in [(0, 0), (1, 2), (2, 1)]:
        Ep = O.energy_from_full(O.Oracle(mol.moved(at, ax, h)).eri_full(), D)[0]
        Em = O.energy_from_full(O.Oracle(mol.moved(at, ax, -h)).eri_full(), D)[0]
        assert abs((Ep - Em) / (2 * h) - g[at, ax]) < 1e-6


def test_gradient_open_shell_hybrid_vs_central_fd():
    """PGet1's full 2-PDM (integral_util/pget1.F90:66-106): CoulFac, ExFac and
    the spin density.  The oracle gradient is the derivative of
    E = coulfac/2 tr(D J[D]) - exfac/4 (tr(D K[D]) + tr(DS K[DS]))."""
    mol = B.small_molecule(3, seed=7)
    o = O.Oracle(mol)
    Ca = B.density_factor(o.nbf, 4, 3)
    Cb = B.density_factor(o.nbf, 3, 5)
    Da, Db = Ca @ Ca.T, Cb @ Cb.T
    D, DS = Da + Db, Da - Db
    cf, xf = 0.9, 0.25
    g = o.grad(D, exfac=xf, coulfac=cf, DS=DS)
    assert np.abs(g.sum(0)).max() < 1e-10

    def energy(eri):
        _, J, K = O.energy_from_full(eri, D)
        KS = np.einsum("acbd,cd->ab", eri, DS)
        return 0.5 * cf * np.sum(D * J) - 0.25 * xf * (np.sum(D * K) + np.sum(DS * KS))

    h = 1e-4
    for at, ax in [(0, 0), (1, 2), (2, 1)]:
        Ep = energy(O.Oracle(mol.moved(at, ax, h)).eri_full())
        Em = energy(O.Oracle(mol.moved(at, ax, -h)).eri_full())
        assert abs((Ep - Em) / (2 * h) - g[at, ax]) < 1e-6
    # linear in the factors
    gJ = o.grad(D, exfac=0.0)
    gK = o.grad(D, exfac=1.0, coulfac=0.0, DS=DS)
    assert np.abs(g - (cf * gJ + xf * gK)).max() < 1e-11 * max(1.0, np.abs(g).max())


def test_scf065_one_electron_pins(scf065):
    """The one-electron oracle against the reference's test 065 checkfile:
    SEWARD_KINETIC / SEWARD_ATTRACT are the first packed element of the
    kinetic and nuclear-attraction matrices (integral_util/oneel.F90:302-303),
    POTNUC the nuclear repulsion; the embedded orbitals are orthonormal."""
    from oracle import oneint
    mol, z, Cocc = scf065["mol"], scf065["z"], scf065["Cocc"]
    S, T, V = oneint.one_electron(mol)
    assert abs(T[0, 0] - z["SEWARD_KINETIC"]) < 1e-10
    assert abs(V[0, 0] - z["SEWARD_ATTRACT"]) < 1e-10
    assert abs(oneint.nuclear_repulsion(mol) - z["POTNUC"]) < 1e-12
    assert np.abs(np.diag(S) - 1.0).max() < 1e-13
    assert np.abs(Cocc.T @ S @ Cocc - np.eye(Cocc.shape[1])).max() < 1e-10


def test_scf065_energy_from_oracle_cholesky(scf065):
    """E_SCF of the reference's test 065 from the oracle's Cholesky vectors
    (ThrCom 1e-4, as Seward's Cholesky keyword sets it).  The reference's own
    harness accepts |dE| <= 1e-4 for this value (tolerance digits 4,
    Tools/pymolcas/check_test.py:137-151); the Cholesky error itself is of
    that order (the exact-ERI energy is 9.4e-5 below E_SCF), so matching the
    printed digits would need the reference's decomposition bit for bit.
    The algorithm-4 defaults (one shell pair per pass, cho_inp.F90:709-715;
    Cho_Qualify_2) land 2.1e-5 from E_SCF.  MXSHPR 0 (algorithms 1-3: shell
    pairs are qualified until MinQual) gives a valid decomposition with fewer
    passes, checked through its residual diagonal."""
    from conftest import rhf_energy
    from oracle import oneint
    mol, z, Cocc = scf065["mol"], scf065["z"], scf065["Cocc"]
    S, T, V = oneint.one_electron(mol)
    D = 2.0 * Cocc @ Cocc.T
    o = O.Oracle(mol)
    res = o.cholesky(thrcom=1e-4)
    J, K = o.cho_jk(res["L"], math.sqrt(2.0) * Cocc)
    E = rhf_energy(T + V, J, K, D, float(z["POTNUC"]))
    print(f"065: E = {E:.12f}  E_SCF = {float(z['E_SCF']):.12f}  dE = {E - float(z['E_SCF']):.2e}")
    assert abs(E - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])
    diag = o.eri_diag()
    for mx, ia in ((1, 1), (0, 2)):
        r = o.cholesky(thrcom=1e-4, mxshpr=mx, ialqua=ia)
        resid = diag - np.einsum("tj,tj->t", r["L"], r["L"])
        assert resid.max() <= 1e-4 and resid.min() > -1e-10, (mx, ia)
        assert len(set(r["piv"].tolist())) == r["M"]
    assert r["npass"] < res["npass"]  # several shell pairs per pass


def test_cholesky_qualify_2_replaces_when_a_shell_pair_exceeds_maxqual():
    """Cho_Qualify_2 (IALQUA 2, the default; cho_qualify_2.F90): once MaxQual
    diagonals of a shell pair are taken, a larger one replaces the smallest.
    With shell pairs of up to 450 AO pairs this changes the pivots relative
    to in-order qualification (Cho_Qualify_1); both are valid decompositions."""
    mol = B.make_molecule("bigpair", 2, [("7s6p5d", 2)], 3)
    o = O.Oracle(mol)
    diag = o.eri_diag()
    a = o.cholesky(thrcom=1e-6, ialqua=1)
    b = o.cholesky(thrcom=1e-6)  # ialqua 2
    assert not (a["M"] == b["M"] and np.array_equal(a["piv"], b["piv"]))
    for r in (a, b):
        resid = diag - np.einsum("tj,tj->t", r["L"], r["L"])
        assert resid.max() <= 1e-6 and resid.min() > -1e-10
        assert len(set(r["piv"].tolist())) == r["M"]


def test_cd_incore_restatement():
    """CD_InCore (cholesky_util/cd_incore_1.F90) restated: a rank-7 PSD matrix
    gives 7 vectors reproducing it, a slightly negative diagonal (above
    ThrNeg's failure bound) is zeroed with its row and column, a diagonal below
    -1e-8 fails with irc 101 and too small a MxVec with irc 102."""
    rng = np.random.default_rng(1)
    C0 = rng.standard_normal((40, 7))
    X = C0 @ C0.T
    V, irc = O.cd_incore(X, 1e-10)
    assert irc == 0 and V.shape == (40, 7)
    assert np.abs(V @ V.T - X).max() < 1e-12 * np.abs(X).max()
    X2 = X.copy()
    X2[3, :] = 0.0
    X2[:, 3] = 0.0
    X2[3, 3] = -5e-12
    V2, irc2 = O.cd_incore(X2, 1e-10)
    assert irc2 == 0 and np.all(V2[3] == 0.0)
    X3 = X.copy()
    X3[5, 5] = -1e-7
    assert O.cd_incore(X3, 1e-10)[1] == 101
    assert O.cd_incore(X, 1e-10, maxvec=3)[1] == 102
