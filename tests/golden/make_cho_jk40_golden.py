"""Generate tests/golden/cho_jk40_oracle.npz: the oracle's pivoted Cholesky
decomposition (algorithm 4 restatement of oracle/oracle.cpp: MXSHPR = 1,
Cho_Qualify_2, CD_InCore_1p, damped Cho_SetRed) of a 497-function molecule
at ThrCom 1e-4, so that a GPU test can compare the device decomposition's
pivot sequence well beyond the 84-function C1 system (the oracle's run takes
tens of minutes, which is why it is stored).

Workload: the 40-atom slice of the 1500-function mix that the J/K tests and
`bench.py --leg jk --natom 40` use (3s2p1d and 2s1p atoms, seed 3).  Stored:
the pivots as AO index pairs (a >= b; independent of the rs numbering), the
pass of each vector, the vector and pass counts, and every vector's sum of
squares.

    python tests/golden/make_cho_jk40_golden.py
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


def molecule():
    """The 40-atom slice of the 1500-function (C3) mix, as bench.py builds it."""
    c3 = B.CONFIGS["c3"]
    natom = 40
    mix = [(t, max(1, round(k * natom / c3["natom"]))) for t, k in c3["mix"]]
    mix[-1] = (mix[-1][0], natom - sum(k for _, k in mix[:-1]))
    return B.make_molecule(f"jk{natom}", natom, mix, c3["seed"])


def main():
    O.build()
    mol = molecule()
    o = O.Oracle(mol)
    t0 = time.time()
    ref = o.cholesky(thrcom=THRCOM, maxvec=4000)
    L = ref["L"]
    a, b, _ = o.rs_list()  # the rs list of this decomposition
    print(f"oracle Cholesky of jk40 ({mol.nbf} functions) at ThrCom {THRCOM}: M = {ref['M']}, "
          f"{ref['npass']} passes, {time.time() - t0:.1f} s on {O.num_threads()} threads")
    np.savez(os.path.join(HERE, "cho_jk40_oracle.npz"), thrcom=THRCOM, nbf=mol.nbf, piv_a=a[ref["piv"]],
             piv_b=b[ref["piv"]],
             pass_of=ref["pass_of"], M=ref["M"], npass=ref["npass"], norm2=(L * L).sum(0))


if __name__ == "__main__":
    main()
