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


def test_jk_mixed_vs_fp64(setup):
    """Mixed path (FP32 vectors, split-BF16 products, FP32 block accumulation,
    FP64 across blocks): error stated against the FP64 path."""
    mol, g, o, ref, Cm = setup
    C = torch.from_numpy(Cm)
    J, K = (x.cpu().numpy() for x in g.cho_jk(C, precision=MolGpu.PREC_FP64))
    Jm, Km = (x.cpu().numpy() for x in g.cho_jk(C, precision=MolGpu.PREC_MIXED))
    D = Cm @ Cm.T
    E = 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K)
    Em = 0.5 * np.sum(D * Jm) - 0.25 * np.sum(D * Km)
    relJ = np.abs(Jm - J).max() / np.abs(J).max()
    relK = np.abs(Km - K).max() / np.abs(K).max()
    print(f"mixed vs fp64: rel J {relJ:.2e}  rel K {relK:.2e}  dE {Em - E:.3e} (E = {E:.6f})")
    assert relJ < 1e-6
    assert relK < 1e-4
    assert abs(Em - E) < 1e-5 * abs(E)


@pytest.mark.parametrize("rank", [1, 17, 300])
def test_jk_mixed_density_ranks(setup, rank):
    """Mixed path at density ranks that exercise a single narrow tensor-core N
    tile, an odd width and two N tiles (rank > 256), against the FP64 path."""
    mol, g, o, ref, _ = setup
    C = torch.from_numpy(B.density_factor(g.nbf, rank, 7))
    J, K = (x.cpu().numpy() for x in g.cho_jk(C, precision=MolGpu.PREC_FP64))
    Jm, Km = (x.cpu().numpy() for x in g.cho_jk(C, precision=MolGpu.PREC_MIXED))
    assert np.abs(Jm - J).max() < 1e-6 * np.abs(J).max()
    assert np.abs(Km - K).max() < 1e-4 * np.abs(K).max()


def test_c1_cluster_jk_energy():
    """C1 (6 atoms, 84 functions, rank-15 density, ThrCom 1e-6): J, K and
    E = 1/2 tr(DJ) - 1/4 tr(DK) of the FP64 path against the oracle's J/K
    from the oracle's own vectors (same pivots), and the mixed path's energy
    error stated against the FP64 path."""
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
    assert abs(Em - E) < 1e-5 * abs(E)


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
