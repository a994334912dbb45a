"""The FP64 work models behind the ERI and gradient roofline figures
(mg_eri_work, mg_drvg1_flops) against the operations the oracle's restated
loops execute for the same quartets (the counting build, see
test_oracle_flops.py).

The oracle contracts each primitive quartet straight into every contracted
output and evaluates Assg1's nine derivative products term by term, the
device kernels factor both; so the models count fewer operations than the
oracle executes.  The bars hold them between a quarter (or a tenth) of the
oracle's count and the count itself (for ERIs per primitive quartet: the
device drops negligible primitive pairs once at set-up, the oracle evaluates
every pair): a model above the count would inflate the achieved FLOP/s, one
far below it would mean it leaves stages out."""
import numpy as np
import pytest

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, unique_quartets

pytestmark = pytest.mark.gpu

CUTINT = 1e-12
ERI_STAGES = ("prim", "roots", "rys2d", "rysef", "contract", "hrr")
GRAD_STAGES = ("prim", "roots", "rys2d", "transfer", "assg1", "pdm")


def _fmt(c):
    return ", ".join(f"{k} {v:.3e}" for k, v in c.items() if v)


def test_eri_work_model_vs_oracle_count():
    """400 seeded quartets of the 40-atom, 600-function uneven-contraction
    workload (the ERI throughput sample's distribution)."""
    mol = B.config_molecule("c2")
    g = MolGpu(mol)
    q = unique_quartets(len(mol.shells), g.schwarz(), CUTINT)
    rng = np.random.default_rng(0)
    sel = q[np.sort(rng.choice(len(q), 400, replace=False))]
    o = O.Oracle(mol, counting=True)
    o.flops(reset=True)
    for i, j, k, l in sel:
        o.eri_quartet(int(i), int(j), int(k), int(l))
    c = o.flops()
    counted = sum(c[s] for s in ERI_STAGES)
    assert counted == sum(c.values())
    pq_dev, model = g.eri_work(sel)
    pq_orc = c["prim"] / 16  # 16 set-up operations per primitive quartet
    per_orc, per_dev = counted / pq_orc, model / pq_dev
    print(f"ERI, 400 quartets: oracle executes {counted:.4e} ({_fmt(c)}) over {pq_orc:.0f} primitive quartets, "
          f"{per_orc:.0f} per primitive quartet; model {model:.4e} = {model / counted:.3f} of it, over the "
          f"{pq_dev:.0f} primitive quartets left after the primitive-pair screening, {per_dev:.0f} per primitive "
          f"quartet ({per_dev / per_orc:.3f})")
    assert model <= counted
    assert pq_dev <= pq_orc
    assert 0.25 * per_orc <= per_dev <= per_orc


@pytest.mark.parametrize("which", ["c4like3", "c4"])
def test_gradient_work_model_vs_oracle_count(which):
    """The 3-atom 4s3p2d cluster over its whole quartet list, and the 20-atom
    460-function gradient workload over every 100th screened quartet (the
    oracle's tally scaled by the number of quartets over the sampled ones)."""
    if which == "c4":
        mol, rank, seed, stride = B.config_molecule("c4"), 40, 4, 100
    else:
        mol, rank, seed, stride = B.make_molecule("c4like", 3, [("4s3p2d", 3)], 4), 6, 3, 1
    g = MolGpu(mol)
    o = O.Oracle(mol, counting=True)
    Cm = B.density_factor(g.nbf, rank, seed)
    D = Cm @ Cm.T
    o.schwarz()  # the screening's own ERIs are not part of the gradient's count
    o.flops(reset=True)
    _, nq = O.grad_sampled(o, D, CUTINT, stride)
    c = o.flops()
    nsamp = (nq + stride - 1) // stride
    counted = sum(c[s] for s in GRAD_STAGES) * nq / nsamp
    assert c["rysef"] == 0 and c["contract"] == 0 and c["hrr"] == 0
    model = g.drvg1_flops(CUTINT)
    print(f"gradient {which}, {nq} quartets (every {stride}th counted): oracle executes {counted:.4e} "
          f"({_fmt(c)}); model {model:.4e} = {model / counted:.3f} of it")
    assert 0.1 * counted <= model <= counted
