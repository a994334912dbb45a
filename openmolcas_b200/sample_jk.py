"""Cholesky J/K of one synthetic cluster (timing and profiling driver).

    python -m openmolcas_b200.sample_jk [natom] [thrcom] [repeats]

Builds `natom` atoms of the 1500-function cluster's basis mix (3s2p1d and
2s1p, as the 120-atom configuration), decomposes the ERI matrix at `thrcom`,
then times the mixed-precision and the FP64 J/K for a rank-200 density.  The
J/K calls run inside an NVTX range named "jk" so that a profiler can select
them (ncu --nvtx --nvtx-include "jk/").
"""
import sys

import torch

from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu


def main(argv):
    natom = int(argv[1]) if len(argv) > 1 else 40
    thrcom = float(argv[2]) if len(argv) > 2 else 1e-6
    reps = int(argv[3]) if len(argv) > 3 else 2
    c3 = B.CONFIGS["c3"]
    mix = [(t, max(1, round(n * natom / c3["natom"]))) for t, n in c3["mix"]]
    mix[-1] = (mix[-1][0], natom - sum(n for _, n in mix[:-1]))
    m = B.make_molecule(f"jk{natom}", natom, mix, c3["seed"])
    g = MolGpu(m)
    info = g.cho_drv(thrcom=thrcom)
    Cm = torch.from_numpy(B.density_factor(m.nbf, min(200, m.nbf // 2), c3["seed"])).cuda()
    out = {}
    for name, prec in (("mixed", MolGpu.PREC_MIXED), ("fp64", MolGpu.PREC_FP64)):
        g.cho_jk(Cm, precision=prec)
        torch.cuda.synchronize()
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            torch.cuda.nvtx.range_push("jk")
            e0.record()
            J, K = g.cho_jk(Cm, precision=prec)
            e1.record()
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
        out[name] = (e0.elapsed_time(e1), J, K)
    relK = float((out["mixed"][2] - out["fp64"][2]).abs().max() / out["fp64"][2].abs().max())
    print(f"jk{natom}: nbf {m.nbf}, M {info['M']}, mixed {out['mixed'][0]:.2f} ms, fp64 {out['fp64'][0]:.2f} ms, "
          f"rel K {relK:.2e}")


if __name__ == "__main__":
    main(sys.argv)
