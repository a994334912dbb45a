"""GPU Cholesky (algorithm 4 semantics) against the CPU oracle: same AO-pair
(rs) ordering, same diagonal, the same pivot sequence and pass structure,
vectors equal to FP64 rounding, and the reconstruction bound of
Cho_X_CheckDiag (|(ab|ab) - sum_J L_ab,J^2| <= ThrCom)."""
import numpy as np
import pytest

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which,thr", [("small", 1e-6), ("c1", 1e-6), ("small", 1e-4)])
def test_cholesky_matches_oracle(which, thr):
    mol = B.small_molecule(3, seed=5) if which == "small" else B.config_molecule("c1")
    g = MolGpu(mol)
    o = O.Oracle(mol)
    info = g.cho_drv(thrcom=thr)
    ref = o.cholesky(thrcom=thr)
    a, b, sp = g.cho_rs_list()
    oa, ob, osp = o.rs_list()
    assert np.array_equal(a, oa) and np.array_equal(b, ob) and np.array_equal(sp, osp)
    d = g.cho_diag().cpu().numpy()
    assert np.abs(d - o.eri_diag()).max() < 1e-11 * max(1.0, np.abs(d).max())
    piv, pas = g.cho_pivots()
    assert info["M"] == ref["M"]
    assert np.array_equal(piv, ref["piv"]), "pivot sequence differs"
    assert np.array_equal(pas, ref["pass_of"])
    L = g.cho_vectors().cpu().numpy().T
    assert np.abs(L - ref["L"]).max() < 1e-9
    rec = (L * L).sum(1)
    assert np.all(o.eri_diag() - rec <= thr * 1.0001)


def test_cholesky_pivots_at_497_functions():
    """A 497-function molecule (the 40-atom slice of the 1500-function mix) at
    ThrCom 1e-4 against the oracle's decomposition of the same molecule, stored
    in tests/golden/cho_jk40_oracle.npz by make_cho_jk40_golden.py (the oracle
    takes minutes): the same vector count and pass structure, the same pivot
    sequence (as AO pairs) and every vector's sum of squares within 1e-10."""
    import os
    import torch
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "cho_jk40_oracle.npz"))
    c3 = B.CONFIGS["c3"]
    natom = 40
    mix = [(t, max(1, round(k * natom / c3["natom"]))) for t, k in c3["mix"]]
    mix[-1] = (mix[-1][0], natom - sum(k for _, k in mix[:-1]))
    mol = B.make_molecule(f"jk{natom}", natom, mix, c3["seed"])
    assert mol.nbf == int(z["nbf"])
    g = MolGpu(mol)
    info = g.cho_drv(thrcom=float(z["thrcom"]))
    assert info["M"] == int(z["M"]) and info["npass"] == int(z["npass"])
    piv, pas = g.cho_pivots()
    a, b, _ = g.cho_rs_list()
    assert np.array_equal(a[piv], z["piv_a"]) and np.array_equal(b[piv], z["piv_b"]), "pivot sequence differs"
    assert np.array_equal(pas, z["pass_of"])
    Lv = g.cho_vectors()
    norm2 = (Lv * Lv).sum(1).cpu().numpy()  # (M, nrs)
    del Lv
    torch.cuda.empty_cache()
    assert np.abs(norm2 - z["norm2"]).max() <= 1e-10 * np.abs(z["norm2"]).max()
