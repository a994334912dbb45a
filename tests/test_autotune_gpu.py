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
from openmolcas_b200.autotune import CANDIDATES
from openmolcas_b200.molgpu import GRAD_TILES


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


def test_committed_tile_table_is_valid():
    if not os.path.exists(GRAD_TILES):
        pytest.skip("no tuned table: the planner's choices apply")
    with open(GRAD_TILES) as f:
        table = json.load(f)
    assert table["classes"], table
    for key, t in table["classes"].items():
        a, b = (int(x) for x in key.split(","))
        assert 1 <= a <= 7 and 1 <= b <= 7
        assert (t["tpq"], t["order"]) in CANDIDATES
        assert t["ms"] < t["planner_ms"]
