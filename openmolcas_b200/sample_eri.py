"""Run a seeded sample of the Schwarz-screened unique shell quartets of one of
the synthetic configurations through the batched ERI entry point (timing and
profiling driver).

    python -m openmolcas_b200.sample_eri c2 20000 [repeats]

The batched calls run inside an NVTX range named "eri" so that a profiler
can select them (ncu --nvtx --nvtx-include "eri/").
"""
import sys
import time

import numpy as np
import torch

from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, unique_quartets


def main(argv):
    cfg = argv[1] if len(argv) > 1 else "c2"
    n = int(argv[2]) if len(argv) > 2 else 20000
    reps = int(argv[3]) if len(argv) > 3 else 2
    m = B.config_molecule(cfg)
    g = MolGpu(m)
    tm = g.schwarz()
    q = unique_quartets(len(m.shells), tm, 1e-12)
    rng = np.random.default_rng(0)
    sel = q[rng.choice(len(q), min(n, len(q)), replace=False)]
    off = g.quartet_offsets(sel)
    out = torch.empty(int(off[-1]), dtype=torch.float64, device="cuda")
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        torch.cuda.nvtx.range_push("eri")
        e0.record()
        g.eri_quartets(sel, out)
        e1.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    print(f"{cfg}: {len(sel)} of {len(q)} quartets, last {ms[-1]:.2f} ms, {len(sel) / ms[-1] * 1e3:.3e} quartets/s")


if __name__ == "__main__":
    main(sys.argv)
