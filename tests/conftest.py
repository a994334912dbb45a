import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmolgpu.so")


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="session")
def scf065():
    """The reference's test 065 (CO, cc-pVDZ, no symmetry, full Cholesky,
    all 7 occupied orbitals frozen so E_SCF is the energy of the embedded
    orbitals), from tests/golden/scf065_co_ccpvdz.npz (made by
    make_scf065_golden.py).  Returns the molecule, the fixture arrays and the
    doubly occupied orbitals (nbf x 7)."""
    import numpy as np

    from openmolcas_b200 import basis as B

    z = dict(np.load(os.path.join(ROOT, "tests", "golden", "scf065_co_ccpvdz.npz")))
    mol = B.molecule_from_arrays("co_ccpvdz", z["coords"], z["charges"], z["shell_atom"], z["shell_l"],
                                 z["shell_nprim"], z["shell_ncontr"], z["exps"], z["coefs"])
    nocc = int(round(z["occupation"].sum() / 2))
    return dict(mol=mol, z=z, Cocc=z["orbitals"][:nocc].T.copy())


def rhf_energy(h, J, K, D, enuc):
    """Closed-shell energy tr(D h) + 1/2 tr(D J) - 1/4 tr(D K) + E_nuc, D = 2 C_occ C_occ^T."""
    import numpy as np
    return float(np.sum(D * h) + 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K) + enuc)


@pytest.fixture(scope="session")
def grad862():
    """The reference's test 862 (water, 6-31G, no symmetry, conventional
    integrals, SCF + Alaska), first geometry, from
    tests/golden/grad862_h2o_631g.npz (made by make_grad862_golden.py)."""
    import numpy as np

    from openmolcas_b200 import basis as B

    z = dict(np.load(os.path.join(ROOT, "tests", "golden", "grad862_h2o_631g.npz")))
    mol = B.molecule_from_arrays("h2o_631g", z["coords"], z["charges"], z["shell_atom"], z["shell_l"],
                                 z["shell_nprim"], z["shell_ncontr"], z["exps"], z["coefs"])
    return dict(mol=mol, z=z, nocc=int(round(float(z["charges"].sum()) / 2)))


def full_eri_from_blocks(mol, quartets, flat, off):
    """Full (ab|cd) tensor from Eval_IJKL-layout blocks of unique quartets
    (i>=j, k>=l, ij>=kl): block = AOInt(nijkl, a, b, c, d) in Fortran order,
    contracted index fastest, AO = shell offset + component * ncontr + k."""
    import numpy as np

    sh = mol.shells
    offs = np.cumsum([0] + [s.nbf for s in sh])
    n = int(offs[-1])
    eri = np.zeros((n, n, n, n))
    for t, (i, j, k, l) in enumerate(np.asarray(quartets)):
        S = [sh[i], sh[j], sh[k], sh[l]]
        nc = [s.ncontr for s in S]
        nm = [s.ncomp for s in S]
        blk = np.asarray(flat[off[t]:off[t + 1]]).reshape(nc + nm, order="F")
        blk = blk.transpose(4, 0, 5, 1, 6, 2, 7, 3).reshape([s.nbf for s in S])
        si = [slice(offs[x], offs[x + 1]) for x in (i, j, k, l)]
        for a, b, c, d, perm in (
            (0, 1, 2, 3, (0, 1, 2, 3)), (1, 0, 2, 3, (1, 0, 2, 3)), (0, 1, 3, 2, (0, 1, 3, 2)),
            (1, 0, 3, 2, (1, 0, 3, 2)), (2, 3, 0, 1, (2, 3, 0, 1)), (3, 2, 0, 1, (3, 2, 0, 1)),
            (2, 3, 1, 0, (2, 3, 1, 0)), (3, 2, 1, 0, (3, 2, 1, 0))):
            eri[si[a], si[b], si[c], si[d]] = blk.transpose(perm)
    return eri


def exact_jk(eri):
    """jk(C) for scf.rhf from a full ERI tensor: J, K of D = C C^T."""
    import numpy as np
    import torch

    def jk(Cf):
        Cn = Cf.detach().cpu().numpy()
        D = Cn @ Cn.T
        return (torch.from_numpy(np.einsum("abcd,cd->ab", eri, D)),
                torch.from_numpy(np.einsum("acbd,cd->ab", eri, D)))
    return jk


@pytest.fixture(params=["scf071_h2o_ccpvtz", "scf004_h2o_anos"])
def refscf(request):
    """Conventional closed-shell SCF cases of the reference: test 071 (water,
    cc-pVTZ, s to f shells, no symmetry) and test 004 (water, ANO-S 3s2p1d /
    2s1p general contractions, C2v in the reference, all atoms here), from
    tests/golden/<name>.npz (made by make_scf071_golden.py and
    make_scf004_golden.py)."""
    return _symgrad_case(request.param)


@pytest.fixture(params=["scf071_h2o_ccpvtz", "scf004_h2o_anos", "scf007_ch2_inline", "scf078_h2o2_631g",
                        "scf090_sto3g", "scf094_hcn_sto3g", "scf095_hcn_sto3g", "scf099_c2h2o3_631g"])
def refscf_all(request):
    """refscf plus the reference's tests 007 (singlet CH2 with an inline
    cc-pVTZ-type basis without f, C2v in the reference; make_scf007_golden.py),
    078 (water dimer, 6-31G), 090 (STO-3G), 094 and 095 (HCN/CNH, STO-3G) and
    099 (1,2-dioxetanone, 6-31G, from its embedded orbitals), the last five
    from XYZ geometries (make_xyz_golden.py)."""
    return _symgrad_case(request.param)


def _symgrad_case(name):
    import numpy as np

    from openmolcas_b200 import basis as B

    z = dict(np.load(os.path.join(ROOT, "tests", "golden", name + ".npz")))
    mol = B.molecule_from_arrays(name, z["coords"], z["charges"], z["shell_atom"], z["shell_l"],
                                 z["shell_nprim"], z["shell_ncontr"], z["exps"], z["coefs"])
    return dict(mol=mol, z=z, nocc=int(round(float(z["charges"].sum()) / 2)))


# function scope: a parametrised fixture of wider scope makes pytest regroup
# the tests that use it across files, out of collection order
@pytest.fixture(params=["grad020_ch4_ccpvdz", "grad023_ch2o2_ccpvdz"])
def symgrad(request):
    """The reference's tests 020 (CH4, cc-pVDZ, generators x z) and 023
    (CH2O2, cc-pVDZ, generator Y): conventional integrals, SCF + Alaska, first
    geometry, expanded to all atoms, from tests/golden/<name>.npz (made by
    make_symgrad_golden.py).  GRAD[i] is the component grad_comp[i] of atom
    grad_atom[i] (the symmetry-allowed components of the unique centres)."""
    return _symgrad_case(request.param)


@pytest.fixture(params=["grad020_ch4_ccpvdz", "grad023_ch2o2_ccpvdz", "grad019_c4h8_sto3g",
                        "grad021_c6h6_sto3g"])
def symgrad_all(request):
    """symgrad plus the reference's tests 019 (C4H8, STO-3G, generators z y x)
    and 021 (benzene, STO-3G, generators x y z), same layout."""
    return _symgrad_case(request.param)
