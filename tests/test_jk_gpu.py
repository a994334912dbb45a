"""J/K from Cholesky vectors on the GPU against the CPU oracle.

FP64 path: vs the oracle's J/K built from the oracle's own vectors (same
pivots, vectors equal to rounding) at 1e-10 relative, and vs exact J/K from
the full ERI tensor within the decomposition error."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    mol = B.small_molecule(3, seed=5)
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-8)
    o = O.Oracle(mol)
    ref = o.cholesky(thrcom=1e-8)
    Cm = B.density_factor(g.nbf, 6, 2)
    return mol, g, o, ref, Cm


def test_jk_fp64_vs_oracle(setup):
    mol, g, o, ref, Cm = setup
    J, K = g.cho_jk(torch.from_numpy(Cm), precision=MolGpu.PREC_FP64)
    Jo, Ko = o.cho_jk(ref["L"], Cm)
    J, K = J.cpu().numpy(), K.cpu().numpy()
    sJ, sK = np.abs(Jo).max(), np.abs(Ko).max()
    assert np.abs(J - Jo).max() < 1e-10 * sJ
    assert np.abs(K - Ko).max() < 1e-10 * sK
    assert np.abs(J - J.T).max() == 0.0 and np.abs(K - K.T).max() == 0.0


def test_jk_fp64_vs_exact_integrals(setup):
    mol, g, o, ref, Cm = setup
    eri = o.eri_full()
    D = Cm @ Cm.T
    E, Je, Ke = O.energy_from_full(eri, D)
    J, K = (x.cpu().numpy() for x in g.cho_jk(torch.from_numpy(Cm), precision=MolGpu.PREC_FP64))
    scale = np.abs(D).sum()
    assert np.abs(J - Je).max() < 1e-8 * scale
    assert np.abs(K - Ke).max() < 1e-8 * scale
    Eg = 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K)
    assert abs(Eg - E) < 1e-7 * scale * scale


# Mixed path bar: the energy difference to the plain FP64 path at most
# 1e-8 Eh (absolute), and K within 1e-10 of the FP64 K relative to its largest
# element (6 slices carry about 47 bits; both paths differ from exact
# arithmetic by FP64 roundings only).  J is FP64 in both paths.
DE_BAR = 1e-8
RELK_BAR = 1e-10
RELJ_BAR = 1e-13


def _jk_pair(g, C, precision=MolGpu.PREC_MIXED):
    J, K = (x.cpu().numpy() for x in g.cho_jk(C, precision=MolGpu.PREC_FP64))
    Jm, Km = (x.cpu().numpy() for x in g.cho_jk(C, precision=precision))
    return J, K, Jm, Km


def _energy(D, J, K):
    return 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K)


def _selftest(g, A, Bm, s):
    import ctypes as C
    from openmolcas_b200.molgpu import lib
    f = lib().mg_sliced_selftest
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 7
    ld, r = A.shape[0], Bm.shape[0]
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major A
    dB = torch.from_numpy(Bm).cuda()                          # column-major B = Bm^T (ld x r)
    X = torch.zeros(r, ld, dtype=torch.float64, device="cuda")  # column-major ld x r
    K = torch.zeros(ld, ld, dtype=torch.float64, device="cuda")
    rc = f(g.h, ld, r, s, dA.data_ptr(), dB.data_ptr(), X.data_ptr(), K.data_ptr(), None, None, None)
    assert rc == 0
    return X.cpu().numpy().T, K.cpu().numpy().T


@pytest.mark.parametrize("ld,r", [(128, 6), (256, 208), (384, 300)])
def test_sliced_engine_on_dense_matrices(setup, ld, r):
    """The 8-bit sliced tensor-core engine (mg_sliced_selftest: X = A B^T, then
    K = X X^T) against FP64 products, on rows with mixed signs, entries near
    the row maximum and round-off-sized entries of either sign (a remainder
    that rounds up to 1 must carry back), at 6 slices: X and the lower
    triangle of K within 1e-11 of their largest elements."""
    g = setup[1]
    rng = np.random.default_rng(ld + r)
    A = rng.standard_normal((ld, ld))
    A[rng.random((ld, ld)) < 0.2] = -1e-31
    A[rng.random((ld, ld)) < 0.05] = 3e-40
    A[:, 0] = -np.abs(A).max(1) * (1 - 2**-40)
    Bm = rng.standard_normal((r, ld))
    Bm[rng.random((r, ld)) < 0.2] = -7e-33
    X, K = _selftest(g, A, Bm, 6)
    Xe = A @ Bm.T
    Ke = X @ X.T
    lo = np.tril_indices(ld)
    assert np.abs(X - Xe).max() < 1e-11 * np.abs(Xe).max()
    assert np.abs(K[lo] - Ke[lo]).max() < 1e-11 * np.abs(Ke).max()


def test_jk_mixed_vs_fp64(setup):
    """Mixed path (FP64 vectors cut into 8-bit slices, exact INT32 tensor-core
    products): J, K and the energy against the FP64 path."""
    mol, g, o, ref, Cm = setup
    J, K, Jm, Km = _jk_pair(g, torch.from_numpy(Cm))
    D = Cm @ Cm.T
    E, Em = _energy(D, J, K), _energy(D, Jm, Km)
    relJ = np.abs(Jm - J).max() / np.abs(J).max()
    relK = np.abs(Km - K).max() / np.abs(K).max()
    print(f"mixed vs fp64: rel J {relJ:.2e}  rel K {relK:.2e}  dE {Em - E:.3e} (E = {E:.6f})")
    assert relJ < RELJ_BAR
    assert relK < RELK_BAR
    assert abs(Em - E) <= DE_BAR
    assert np.abs(Km - Km.T).max() == 0.0


def test_jk_sliced_error_falls_with_slices(setup):
    """Each added 8-bit slice cuts the exchange error by about 2^8: the error
    of K against the FP64 path falls by at least 30x per slice from 3 to 6
    slices (MG_PREC_SLICED(s))."""
    mol, g, o, ref, Cm = setup
    C = torch.from_numpy(Cm)
    K = g.cho_jk(C, precision=MolGpu.PREC_FP64)[1].cpu().numpy()
    errs = []
    for s in (3, 4, 5, 6):
        Ks = g.cho_jk(C, precision=MolGpu.PREC_SLICED(s))[1].cpu().numpy()
        errs.append(np.abs(Ks - K).max() / np.abs(K).max())
    print("rel K error vs slices 3..6:", ", ".join(f"{e:.2e}" for e in errs))
    for a, b in zip(errs, errs[1:]):
        assert b < a / 30.0 or b < 1e-14


@pytest.mark.parametrize("rank", [1, 17, 300])
def test_jk_mixed_density_ranks(setup, rank):
    """Mixed path at density ranks that exercise a single narrow tensor-core N
    tile, an odd width and two N tiles (rank > 256), against the FP64 path."""
    mol, g, o, ref, _ = setup
    Cn = B.density_factor(g.nbf, rank, 7)
    J, K, Jm, Km = _jk_pair(g, torch.from_numpy(Cn))
    D = Cn @ Cn.T
    assert np.abs(Jm - J).max() < RELJ_BAR * np.abs(J).max()
    assert np.abs(Km - K).max() < RELK_BAR * np.abs(K).max()
    assert abs(_energy(D, Jm, Km) - _energy(D, J, K)) <= DE_BAR


def test_jk_mixed_many_vector_blocks():
    """40 atoms of the 1500-function cluster's basis mix (497 functions,
    ThrCom 1e-6: 4281 vectors, so 67 blocks of 64 vectors in 5 exchange-product
    groups and a short last block), rank-200 density: mixed against FP64 at
    the same bars."""
    c3 = B.CONFIGS["c3"]
    natom = 40
    mix = [(t, max(1, round(k * natom / c3["natom"]))) for t, k in c3["mix"]]
    mix[-1] = (mix[-1][0], natom - sum(k for _, k in mix[:-1]))
    mol = B.make_molecule(f"jk{natom}", natom, mix, c3["seed"])
    g = MolGpu(mol)
    info = g.cho_drv(thrcom=1e-6)
    assert info["M"] % 64 != 0 and info["M"] > 16 * 64
    Cn = B.density_factor(g.nbf, 200, c3["seed"])
    J, K, Jm, Km = _jk_pair(g, torch.from_numpy(Cn))
    D = Cn @ Cn.T
    E, Em = _energy(D, J, K), _energy(D, Jm, Km)
    relK = np.abs(Km - K).max() / np.abs(K).max()
    print(f"jk40: nbf {g.nbf} M {info['M']} rel K {relK:.2e} dE {Em - E:.2e} (E = {E:.6f})")
    assert np.abs(Jm - J).max() < RELJ_BAR * np.abs(J).max()
    assert relK < RELK_BAR
    assert abs(Em - E) <= DE_BAR


def test_jk_mixed_general_contraction():
    """Generally contracted shells of every l (an ANO-like 9s5p4d -> 4s3p2d
    set on one atom, narrower shells on two more), whose AO ranges straddle
    the 16-row blocks in which the slicing kernel unpacks the rs-packed
    vectors into squares, ThrCom 1e-6, rank-10 density: mixed against FP64
    at the same bars."""
    rng = np.random.default_rng(21)
    coords = np.array([[0.0, 0.0, 0.0], [1.9, 0.4, -0.3], [-0.7, 2.1, 0.8]])
    sh = [(0, 2, 4, 2), (0, 0, 9, 4), (0, 1, 5, 3), (1, 0, 6, 2), (1, 1, 3, 1), (2, 0, 3, 2), (2, 2, 2, 1)]
    exps, coefs = [], []
    for _, l, npr, nco in sh:
        exps += list(0.1 * 2.7 ** np.arange(npr))
        coefs += list(rng.standard_normal(npr * nco))
    mol = B.molecule_from_arrays("general", coords, [6.0, 1.0, 1.0], [x[0] for x in sh], [x[1] for x in sh],
                                 [x[2] for x in sh], [x[3] for x in sh], exps, coefs)
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-6)
    Cn = B.density_factor(g.nbf, 10, 5)
    J, K, Jm, Km = _jk_pair(g, torch.from_numpy(Cn))
    D = Cn @ Cn.T
    assert np.abs(Jm - J).max() < RELJ_BAR * np.abs(J).max()
    assert np.abs(Km - K).max() < RELK_BAR * np.abs(K).max()
    assert abs(_energy(D, Jm, Km) - _energy(D, J, K)) <= DE_BAR


def test_c1_cluster_jk_energy():
    """C1 (6 atoms, 84 functions, rank-15 density, ThrCom 1e-6): J, K and
    E = 1/2 tr(DJ) - 1/4 tr(DK) of the FP64 path against the oracle's J/K
    from the oracle's own vectors (same pivots), and the mixed path's energy
    within 1e-8 Eh of the FP64 path's."""
    mol = B.config_molecule("c1")
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-6)
    o = O.Oracle(mol)
    ref = o.cholesky(thrcom=1e-6)
    Cm = B.density_factor(g.nbf, B.CONFIGS["c1"]["rank"], B.CONFIGS["c1"]["seed"])
    J, K = (x.cpu().numpy() for x in g.cho_jk(torch.from_numpy(Cm), precision=MolGpu.PREC_FP64))
    Jo, Ko = o.cho_jk(ref["L"], Cm)
    assert np.abs(J - Jo).max() < 1e-10 * np.abs(Jo).max()
    assert np.abs(K - Ko).max() < 1e-10 * np.abs(Ko).max()
    D = Cm @ Cm.T
    E = 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K)
    Eo = 0.5 * np.sum(D * Jo) - 0.25 * np.sum(D * Ko)
    assert abs(E - Eo) < 1e-10 * abs(Eo)
    Jm, Km = (x.cpu().numpy() for x in g.cho_jk(torch.from_numpy(Cm), precision=MolGpu.PREC_MIXED))
    Em = 0.5 * np.sum(D * Jm) - 0.25 * np.sum(D * Km)
    print(f"C1: E = {E:.10f}, |E - E_oracle| = {abs(E - Eo):.2e}, mixed dE = {Em - E:.2e}")
    assert abs(Em - E) <= DE_BAR


def test_scf065_energy_through_device_cholesky(scf065):
    """The reference's test 065 (CO, cc-pVDZ) through the device path: Cho_Drv
    at ThrCom 1e-4 (mg_cho_drv) and FP64 J/K (mg_cho_jk) for the embedded
    orbitals, with the oracle's one-electron matrices.  The energy equals the
    oracle's from its own vectors (same pivots) to 1e-9 and E_SCF within the
    reference harness's own tolerance for it (10^-4, the checkfile's digits)."""
    from conftest import rhf_energy
    from oracle import oneint
    mol, z, Cocc = scf065["mol"], scf065["z"], scf065["Cocc"]
    S, T, V = oneint.one_electron(mol)
    D = 2.0 * Cocc @ Cocc.T
    Cm = np.sqrt(2.0) * Cocc
    g = MolGpu(mol)
    g.cho_drv(thrcom=1e-4)
    piv, _ = g.cho_pivots()
    J, K = (x.cpu().numpy() for x in g.cho_jk(torch.from_numpy(Cm), precision=MolGpu.PREC_FP64))
    E = rhf_energy(T + V, J, K, D, float(z["POTNUC"]))
    o = O.Oracle(mol)
    ref = o.cholesky(thrcom=1e-4)
    Jo, Ko = o.cho_jk(ref["L"], Cm)
    Eo = rhf_energy(T + V, Jo, Ko, D, float(z["POTNUC"]))
    print(f"065 device: E = {E:.12f}  oracle {Eo:.12f}  E_SCF {float(z['E_SCF']):.12f}")
    assert np.array_equal(piv, ref["piv"])
    assert abs(E - Eo) < 1e-9
    assert abs(E - float(z["E_SCF"])) <= 10.0 ** -int(z["E_SCF_digits"])


@pytest.mark.parametrize("prec", [MolGpu.PREC_FP64, MolGpu.PREC_MIXED])
def test_jk_batch_equals_single_calls(setup, prec):
    """mg_cho_jk_batch (three densities of different rank in one pass over the
    vectors) equals one mg_cho_jk per density, J and K within 1e-13 of their
    largest elements, both paths (not to the bit: the CTA tiles of K and the
    Coulomb contractions are added with FP64 atomics, whose order varies from
    call to call)."""
    g = setup[1]
    Cs = [torch.from_numpy(B.density_factor(g.nbf, rk, 10 + rk)) for rk in (3, 7, 12)]
    batch = g.cho_jk_batch(Cs, precision=prec)
    for Cf, (Jb, Kb) in zip(Cs, batch):
        J, K = g.cho_jk(Cf, precision=prec)
        assert float((Jb - J).abs().max()) < 1e-13 * float(J.abs().max())
        assert float((Kb - K).abs().max()) < 1e-13 * float(K.abs().max())
