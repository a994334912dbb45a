"""Gradient tile tuning: every tile choice the autotuner can pick gives the
same gradient as the planner's own; the profiled launch (classes one after
another, timed per class) gives the same gradient too; and the committed
table (openmolcas_b200/grad_tiles.json) only names valid choices."""
import json
import os

import numpy as np
import pytest
import torch

from openmolcas_b200 import basis as B
from openmolcas_b200.autotune import CANDIDATES, ERI_CANDIDATES
from openmolcas_b200.molgpu import ERI_TILES, GRAD_TILES


def _setup():
    from openmolcas_b200.molgpu import MolGpu
    mol = B.make_molecule("c4like", 3, [("4s3p2d", 3)], 4)
    g = MolGpu(mol, grad_tiles=None)
    Cm = B.density_factor(g.nbf, 6, 3)
    return g, torch.from_numpy(Cm @ Cm.T)


@pytest.mark.gpu
def test_every_tile_choice_gives_the_same_gradient():
    g, D = _setup()
    ref = g.drvg1(D).cpu().numpy()
    scale = np.abs(ref).max()
    plans = set()
    for tpq, order in CANDIDATES:
        for a in range(1, 8):
            for b in range(1, 8):
                g.set_grad_tile(a, b, tpq, order)
        got = g.drvg1(D).cpu().numpy()
        plans.add(tuple(sorted(g.grad_plan_info().items())))
        assert np.abs(got - ref).max() < 1e-12 * scale, (tpq, order)
    assert len(plans) > 1  # the choices do change the tiles


@pytest.mark.gpu
def test_profiled_gradient_times_every_class():
    g, D = _setup()
    ref = g.drvg1(D).cpu().numpy()
    g.grad_profile(True)
    got = g.drvg1(D).cpu().numpy()
    times = g.grad_class_times()
    plan = g.grad_plan_info()
    assert set(times) == set(plan) and len(times) > 1
    assert all(t > 0 for t in times.values())
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
    g.grad_profile(False)
    assert g.grad_class_times() == {}


@pytest.mark.gpu
def test_every_eri_tile_choice_gives_the_same_integrals():
    """Every class of the s..f test molecule under each ERI candidate, also
    profiled (classes one after another, timed per class)."""
    from openmolcas_b200.molgpu import MolGpu, unique_quartets
    mol = B.small_molecule(3, seed=5)
    g = MolGpu(mol, eri_tiles=None)
    q = unique_quartets(len(mol.shells))
    ref, _ = g.eri_quartets(q)
    ref = ref.cpu().numpy()
    scale = np.abs(ref).max()
    plans = set()
    g.eri_profile(True)
    for tpq, order in ERI_CANDIDATES:
        for a in range(8):
            for b in range(8):
                g.set_eri_tile(a, b, tpq, order)
        got, _ = g.eri_quartets(q)
        times = g.eri_class_times()
        plans.add(tuple(sorted((k, pl) for k, (_, pl) in times.items())))
        assert all(t > 0 for t, _ in times.values()) and len(times) > 1
        assert np.abs(got.cpu().numpy() - ref).max() < 1e-11 * max(1.0, scale), (tpq, order)
    assert len(plans) > 1


@pytest.mark.parametrize("path,cands,lo", [(GRAD_TILES, CANDIDATES, 1), (ERI_TILES, ERI_CANDIDATES, 0)])
def test_committed_tile_tables_are_valid(path, cands, lo):
    if not os.path.exists(path):
        pytest.skip("no tuned table: the planner's choices apply")
    with open(path) as f:
        table = json.load(f)
    for key, t in table["classes"].items():
        a, b = (int(x) for x in key.split(","))
        assert lo <= a <= 7 and lo <= b <= 7
        assert (t["tpq"], t["order"]) in cands
        assert t["ms"] < t["planner_ms"]


def test_pick_keeps_only_clear_wins():
    """The tuner's per-class choice on made-up timings: the fastest candidate
    wins only when it beats the planner by more than the margin, and a class
    one candidate did not time is judged on the others."""
    from openmolcas_b200.autotune import pick
    base = {(3, 3): 100.0, (4, 4): 50.0, (2, 2): 10.0}
    plan = {(3, 3): (128, 8, 1, 3), (4, 4): (256, 4, 1, 4), (2, 2): (128, 16, 2, 2)}
    runs = {
        (256, 1): ({(3, 3): 90.0, (4, 4): 49.5, (2, 2): 11.0},
                   {(3, 3): (256, 16, 2, 1), (4, 4): (256, 8, 1, 1), (2, 2): (256, 16, 4, 1)}),
        (512, 0): ({(3, 3): 95.0, (2, 2): 9.0},
                   {(3, 3): (512, 8, 2, 3), (2, 2): (512, 16, 8, 2)}),
    }
    got = pick(base, plan, runs, 0.02)
    assert set(got) == {"3,3", "2,2"}  # (4,4): 1 % better only
    assert got["3,3"]["tpq"] == 256 and got["3,3"]["order"] == 1 and got["3,3"]["tile"] == [256, 16, 2, 1]
    assert got["3,3"]["ms"] == 90.0 and got["3,3"]["planner_ms"] == 100.0
    assert got["2,2"]["tpq"] == 512 and got["2,2"]["planner_tile"] == [128, 16, 2, 2]
    assert pick(base, plan, runs, 0.2) == {}
