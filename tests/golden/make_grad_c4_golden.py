"""Generate tests/golden/grad_c4_oracle.npz: the oracle's two-electron
gradient (the Drvg1 restatement of oracle/oracle.cpp, FP64, OpenMP) of the
bench's gradient workload, so that a GPU test can compare the device
gradient with the oracle on the full-size workload instead of a slice.

Workload: 20 seeded atoms with 4s3p2d contracted from 8s5p3d primitives
(460 functions, openmolcas_b200.basis.config_molecule("c4")), density
D = C C^T with the seeded rank-40 factor density_factor(nbf, 40, 4), shell
quartets screened at Schwarz 1e-12.  The full oracle gradient takes several
minutes on a few cores, which is why it is stored rather than recomputed.
Stored: the gradient (natom x 3), the screening threshold, and checksums of D
(sum, sum of squares, trace) so the test can confirm it rebuilt the same input.

    python tests/golden/make_grad_c4_golden.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from openmolcas_b200 import basis as B  # noqa: E402

CUTINT = 1e-12


def main():
    O.build()
    cfg = B.CONFIGS["c4"]
    mol = B.config_molecule("c4")
    Cm = B.density_factor(mol.nbf, cfg["rank"], cfg["seed"])
    D = Cm @ Cm.T
    o = O.Oracle(mol)
    o.schwarz()
    t0 = time.time()
    g = o.grad(D, cutint=CUTINT)
    print(f"oracle gradient of c4 ({mol.nbf} functions): {time.time() - t0:.1f} s on {O.num_threads()} threads, "
          f"max |F| {np.abs(g).max():.6f}, |sum F| {np.abs(g.sum(0)).max():.2e}")
    np.savez(os.path.join(HERE, "grad_c4_oracle.npz"), grad=g, cutint=CUTINT,
             d_sum=D.sum(), d_sumsq=(D * D).sum(), d_trace=np.trace(D), nbf=mol.nbf)


if __name__ == "__main__":
    main()
