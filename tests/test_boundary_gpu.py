"""The drop-in entry points beside the batched ones, called through the C ABI:
the per-quartet Do_TwoEl shim (mg_twoel_nosym, integral_util/eval_ijkl.F90:
93-95 with integral_util/twoel_interface.fh), the accumulating CHO_LK_SCF
form (mg_cho_lk_scf, fock_util/cho_lk_scf.F90:14), Cho_Drv's return codes
(cholesky_util/cho_drv_inner.F90:14-19) and the torch.ops.molgpu operators."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import ChoCfg, MolGpu, lib

pytestmark = pytest.mark.gpu

NSD = 20  # iSD4(0:nSD, 4) as Def_Shells fills it (integral_util/def_shells.F90:108-148)


@pytest.fixture(scope="module")
def small():
    mol = B.small_molecule(3, seed=5)
    return mol, MolGpu(mol), O.Oracle(mol).eri_full()


def _isd4(mol, shells):
    isd = np.zeros((4, NSD + 1), dtype=np.int64)  # column-major iSD4(0:nSD, 4): one row per shell here
    for x, s in enumerate(shells):
        sh = mol.shells[s]
        isd[x, 0] = s + 1
        isd[x, 1] = sh.l
        isd[x, 2] = sh.ncomp
        isd[x, 3] = sh.ncontr
        isd[x, 5] = len(sh.exps)
        isd[x, 20] = s + 1
    return isd


def _twoel(g, mol, shells, coor=None, nwork=None):
    f = lib().mg_twoel_nosym
    f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
    if coor is None:
        coor = np.array([mol.shells[s].center for s in shells], dtype=np.float64)
    coor = np.ascontiguousarray(coor, dtype=np.float64)
    nijkl = int(np.prod([mol.shells[s].ncontr for s in shells]))
    nabcd = int(np.prod([mol.shells[s].ncomp for s in shells]))
    wrk = np.full(nijkl * nabcd if nwork is None else nwork, np.nan)
    isd = _isd4(mol, shells)
    noints = C.c_int(1)
    rc = f(g.h, coor.ctypes.data, C.byref(noints), wrk.ctypes.data, wrk.size, isd.ctypes.data, NSD)
    return rc, noints.value, wrk


def _expected_block(mol, eri, shells):
    offs = np.cumsum([0] + [s.nbf for s in mol.shells])
    S = [mol.shells[s] for s in shells]
    nb = [s.ncontr for s in S]
    nm = [s.ncomp for s in S]
    out = np.empty(int(np.prod(nb) * np.prod(nm)))
    nijkl = int(np.prod(nb))
    for m3 in range(nm[3]):
        for m2 in range(nm[2]):
            for m1 in range(nm[1]):
                for m0 in range(nm[0]):
                    c = m0 + nm[0] * (m1 + nm[1] * (m2 + nm[2] * m3))
                    for k3 in range(nb[3]):
                        for k2 in range(nb[2]):
                            for k1 in range(nb[1]):
                                for k0 in range(nb[0]):
                                    ij = k0 + nb[0] * (k1 + nb[1] * (k2 + nb[2] * k3))
                                    a = [offs[s] + m * n + k for s, m, n, k in
                                         zip(shells, (m0, m1, m2, m3), nb, (k0, k1, k2, k3))]
                                    out[ij + nijkl * c] = eri[a[0], a[1], a[2], a[3]]
    return out


@pytest.mark.parametrize("shells", [(0, 0, 0, 0), (2, 1, 3, 0), (1, 3, 0, 2), (3, 3, 1, 2), (0, 4, 4, 1)])
def test_twoel_nosym_any_shell_order(small, shells):
    """Do_TwoEl's layout Wrk(nijkl, iCmp1..4) for shells in any order (the
    shim computes the canonical quartet and transposes the block back)."""
    mol, g, eri = small
    shells = tuple(s % len(mol.shells) for s in shells)
    rc, noints, wrk = _twoel(g, mol, shells)
    assert rc == 0, lib().mg_last_error(g.h)
    assert noints == 0
    ref = _expected_block(mol, eri, shells)
    assert np.abs(wrk - ref).max() <= O.ERI_ABS_TOL


def test_twoel_nosym_rejects_bad_calls(small):
    mol, g, _ = small
    shells = (1, 0, 2, 0)
    coor = np.array([mol.shells[s].center for s in shells])
    coor[2, 1] += 0.5
    assert _twoel(g, mol, shells, coor=coor)[0] == 1  # Coor differs from the shell centres
    assert _twoel(g, mol, shells, nwork=1)[0] == 1     # Wrk too small


def test_cho_lk_scf_accumulates_into_flt(small):
    """FLT += J - FactXI K (CHO_LK_SCF accumulates into FLT and, with -FactXI,
    into KLT which it then adds to FLT): against mg_cho_jk, both precisions."""
    mol, g, _ = small
    g.cho_drv(thrcom=1e-8)
    Cn = torch.from_numpy(B.density_factor(g.nbf, 5, 3)).cuda()
    Cc = Cn.t().contiguous()
    f = lib().mg_cho_lk_scf
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    for prec in (MolGpu.PREC_FP64, MolGpu.PREC_MIXED):
        J, K = g.cho_jk(Cn, precision=prec)
        F0 = torch.randn(g.nbf, g.nbf, dtype=torch.float64, device="cuda")
        F = F0.clone()
        for _ in range(2):
            rc = f(g.h, Cc.data_ptr(), 5, 0.5, F.data_ptr(), prec, None)
            assert rc == 0, lib().mg_last_error(g.h)
        torch.cuda.synchronize()
        ref = F0 + 2.0 * (J - 0.5 * K)
        assert float((F - ref).abs().max()) <= 1e-12 * float(ref.abs().max())


def test_cho_drv_return_codes(small):
    """Cho_Drv's iReturn: 0 decomposed, 1 not decomposed (here: an invalid
    threshold), 2 the vectors do not fit (here: MaxVec too small)."""
    mol, g, _ = small
    f = lib().mg_cho_drv
    cfg = ChoCfg()
    lib().mg_cho_default(C.byref(cfg))
    cfg.thrcom = 1e-6
    assert f(g.h, C.byref(cfg), None) == 0
    cfg.maxvec = 3
    assert f(g.h, C.byref(cfg), None) == 2
    cfg.maxvec = 0
    cfg.thrcom = -1.0
    assert f(g.h, C.byref(cfg), None) == 1


def test_torch_ops(small):
    """torch.ops.molgpu.{eri_batch, cholesky, jk, jk_energy} equal the MolGpu
    calls; jk_energy's backward is dE/dC = 2 (J - K/2) C."""
    from openmolcas_b200 import torch_ops
    from openmolcas_b200.molgpu import unique_quartets
    mol, g, _ = small
    h = torch_ops.register(g)
    q = unique_quartets(len(mol.shells))[:50]
    blocks, off = torch.ops.molgpu.eri_batch(h, torch.from_numpy(q))
    ref, roff = g.eri_quartets(q)
    assert np.array_equal(off.numpy(), roff) and torch.equal(blocks, ref)
    info = torch.ops.molgpu.cholesky(h, 1e-8, 1e-2, 50, 100)
    assert info.tolist() == [g.cho_info()[k] for k in ("nrs", "M", "npass")]
    Cn = torch.from_numpy(B.density_factor(g.nbf, 4, 9)).cuda()
    J, K = torch.ops.molgpu.jk(h, Cn, MolGpu.PREC_FP64)
    Jr, Kr = g.cho_jk(Cn, precision=MolGpu.PREC_FP64)
    assert torch.equal(J, Jr) and torch.equal(K, Kr)
    Cg = Cn.clone().requires_grad_()
    E = torch.ops.molgpu.jk_energy(h, Cg, MolGpu.PREC_FP64)
    E.backward()
    D = Cn @ Cn.t()
    assert abs(float(E) - float(0.5 * (D * J).sum() - 0.25 * (D * K).sum())) < 1e-10 * abs(float(E))
    assert float((Cg.grad - 2.0 * (J - 0.5 * K) @ Cn).abs().max()) < 1e-12 * float(Cg.grad.abs().max())
    torch_ops.unregister(h)


@pytest.mark.parametrize("n,rank,case", [(120, 15, "plain"), (300, 40, "zeroed"), (64, 64, "full"),
                                         (50, 10, "fail"), (50, 10, "maxvec")])
def test_cd_incore_matches_oracle(small, n, rank, case):
    """mg_cd_incore (CD_InCore, cholesky_util/cd_incore.F90:14) against the
    oracle's restatement: the same number of vectors in the same pivot order
    (vectors equal to FP64 rounding), the reconstruction, and the return codes
    101 (a diagonal below -1e-8) and 102 (MxVec too small)."""
    g = small[1]
    rng = np.random.default_rng(n + rank)
    C0 = rng.standard_normal((n, rank))
    X = C0 @ C0.T
    maxvec = None
    if case == "zeroed":  # a diagonal just below zero: zeroed with its row and column
        X[7, :] = 0.0
        X[:, 7] = 0.0
        X[7, 7] = -5e-12
    elif case == "fail":
        X[4, 4] = -1e-6
    elif case == "maxvec":
        maxvec = rank - 3
    Vr, ircr = O.cd_incore(X, 1e-9, maxvec)
    V, irc = g.cd_incore(torch.from_numpy(X), 1e-9, maxvec)
    assert irc == ircr
    V = V.cpu().numpy()
    assert V.shape == Vr.shape
    if V.size:
        assert np.abs(V - Vr).max() < 1e-10 * np.abs(Vr).max()
    if case in ("plain", "zeroed", "full"):
        assert irc == 0 and V.shape[1] == rank
        assert np.abs(V @ V.T - X).max() < 1e-9 * np.abs(X).max()


def test_choscf_lk_decomposes_the_density(small):
    """mg_choscf_lk (ChoSCF_Drv with a decomposed density, scf/choscf_drv.F90:
    99-135): the density is cut into its Cholesky vectors (as many as its
    rank) and FLT += J - FactXI K equals mg_cho_lk_scf with the factor the
    density was made from, both precisions."""
    mol, g, _ = small
    g.cho_drv(thrcom=1e-8)
    Cn = torch.from_numpy(B.density_factor(g.nbf, 5, 3)).cuda()
    D = Cn @ Cn.t()
    Cc = Cn.t().contiguous()
    f = lib().mg_cho_lk_scf
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    for prec in (MolGpu.PREC_FP64, MolGpu.PREC_MIXED):
        F0 = torch.randn(g.nbf, g.nbf, dtype=torch.float64, device="cuda")
        Fa = F0.clone()
        nv = g.choscf_lk(D, 0.5, Fa, precision=prec)
        Fb = F0.clone()
        assert f(g.h, Cc.data_ptr(), 5, 0.5, Fb.data_ptr(), prec, None) == 0
        torch.cuda.synchronize()
        assert nv == 5
        assert float((Fa - Fb).abs().max()) <= 1e-11 * float((Fb - F0).abs().max())
