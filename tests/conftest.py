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
