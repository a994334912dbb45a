"""Generate tests/golden/cho_c2_oracle.npz: the oracle's pivoted Cholesky
decomposition (algorithm 4 restatement of oracle/oracle.cpp: MXSHPR = 1,
Cho_Qualify_2, CD_InCore_1p, damped Cho_SetRed) of the 600-function
uneven-class cluster at ThrCom 1e-4, so that a GPU test can compare the
device decomposition's pivot sequence at that size (the oracle's run takes
minutes on a few cores, which is why it is stored).

Workload: openmolcas_b200.basis.config_molecule("c2") (40 seeded atoms, 2s1p
and 4s3p2d1f shells with 1-12 primitives).  Stored: the pivots (rs index of
each vector's pivot), the pass of each vector, the vector count, the pass
count and every vector's sum of squares (a size-independent fingerprint of
the vectors themselves, which are several GB).

    python tests/golden/make_cho_c2_golden.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from openmolcas_b200 import basis as B  # noqa: E402

THRCOM = 1e-4


def main():
    O.build()
    mol = B.config_molecule("c2")
    o = O.Oracle(mol)
    t0 = time.time()
    ref = o.cholesky(thrcom=THRCOM, maxvec=6000)
    L = ref["L"]
    print(f"oracle Cholesky of c2 ({mol.nbf} functions) at ThrCom {THRCOM}: M = {ref['M']}, "
          f"{ref['npass']} passes, {time.time() - t0:.1f} s on {O.num_threads()} threads")
    np.savez(os.path.join(HERE, "cho_c2_oracle.npz"), thrcom=THRCOM, nbf=mol.nbf, piv=ref["piv"],
             pass_of=ref["pass_of"], M=ref["M"], npass=ref["npass"], norm2=(L * L).sum(0))


if __name__ == "__main__":
    main()
