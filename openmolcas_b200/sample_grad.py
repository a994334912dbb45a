"""Run the two-electron gradient of one synthetic configuration (timing and
profiling driver).

    python -m openmolcas_b200.sample_grad c4 [repeats]
    python -m openmolcas_b200.sample_grad small [repeats]     # 4 atoms of 4s3p2d
    python -m openmolcas_b200.sample_grad medium [repeats]    # 8 atoms of 4s3p2d
"""
import sys

import torch

from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu


def main(argv):
    cfg = argv[1] if len(argv) > 1 else "c4"
    reps = int(argv[2]) if len(argv) > 2 else 2
    if cfg == "small":
        m = B.make_molecule("small4s3p2d", 4, [("4s3p2d", 4)], 4)
        rank = 10
    elif cfg == "medium":
        m = B.make_molecule("medium4s3p2d", 8, [("4s3p2d", 8)], 4)
        rank = 20
    else:
        m = B.config_molecule(cfg)
        rank = B.CONFIGS[cfg]["rank"] or 40
    g = MolGpu(m)
    C = B.density_factor(m.nbf, rank, 4)
    D = torch.from_numpy(C @ C.T).cuda()
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        grad = g.drvg1(D, cutint=1e-12)
        e1.record()
        torch.cuda.synchronize()
    print(f"{cfg}: nbf {m.nbf}, gradient {e0.elapsed_time(e1):.1f} ms, |sum F| = {float(grad.sum(0).abs().max()):.2e}")


if __name__ == "__main__":
    main(sys.argv)
