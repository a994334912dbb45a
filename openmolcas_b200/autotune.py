"""Tile autotuner of the two-electron gradient (mg_drvg1) and of the ERI
batches (mg_eri_quartets).

Both run one persistent kernel per shell-quartet class.  How each class
tiles its work -- threads per work-item group and which dimension of the
primitive-quartet tile (ket primitives, bra primitives and, for the
gradient, roots per wave) shrinks first to fit shared memory -- is chosen by
the planners from a fixed rule.  This tool measures instead: every candidate
(group size x shrink order) is applied to all classes, the work runs
profiled (classes one after another on one stream, an event pair around
each kernel), and each class keeps the candidate with the shortest kernel
time if it beats the planner's own choice by more than the margin.  The
results are written to grad_tiles.json and eri_tiles.json, which MolGpu
applies at handle creation (mg_grad_set_tile, mg_eri_set_tile).

    python -m openmolcas_b200.autotune [--only grad|eri] [--cfg c4] [--eri-cfg c2] [--reps 2]
                                       [--margin 0.02] [--out PATH] [--eri-out PATH]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import ERI_TILES, GRAD_TILES, MolGpu, unique_quartets

# gradient: group size x shrink order (0 ket primitives, 1 roots per wave, 2 bra
# primitives; 3..5 the same from the larger 32 x 16 tile caps)
CANDIDATES = [(tpq, order) for tpq in (128, 256, 512) for order in range(6)]
# ERIs: group size x order = shrink order (0 ket, 1 bra primitives) + 2 (64 x 16 tile caps)
ERI_CANDIDATES = [(tpq, order) for tpq in (64, 128, 256, 512) for order in range(4)]
CUTINT = 1e-12
ERI_SAMPLE = 2_000_000  # the seeded quartet sample of the ERI throughput benchmark


def pick(base, base_plan, runs, margin):
    """Per-class choice: `base` maps a class to the planner's time, `runs`
    maps each candidate to (times, plans) per class.  A class takes the
    candidate with the shortest time when that beats the planner's by more
    than `margin` (a fraction); the entry records the candidate, the tile it
    produced and both times.  Classes a candidate did not time are skipped
    for that candidate."""
    classes = {}
    for k, tb in sorted(base.items()):
        timed = [(r[0][k], cand, r[1][k]) for cand, r in runs.items() if k in r[0]]
        if not timed:
            continue
        tt, (tpq, order), plan = min(timed, key=lambda x: x[0])
        if tt < (1.0 - margin) * tb:
            classes[f"{k[0]},{k[1]}"] = {"tpq": tpq, "order": order, "tile": list(plan), "ms": round(tt, 3),
                                         "planner_tile": list(base_plan[k]), "planner_ms": round(tb, 3)}
    return classes


def _class_times(g, D, reps):
    """Per-class minimum kernel milliseconds over `reps` profiled gradients
    (after one more profiled gradient that re-plans and warms up)."""
    g.drvg1(D, CUTINT)
    torch.cuda.synchronize()
    best = {}
    for _ in range(reps):
        g.drvg1(D, CUTINT)
        for k, t in g.grad_class_times().items():
            best[k] = min(best.get(k, float("inf")), t)
    return best, g.grad_plan_info()


def _set_all(g, tpq, order):
    for a in range(1, 8):
        for b in range(1, 8):
            g.set_grad_tile(a, b, tpq, order)


def _gradient_ms(g, D, reps):
    """Mean device milliseconds of the normal (multi-stream) gradient."""
    g.grad_profile(False)
    g.drvg1(D, CUTINT)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.drvg1(D, CUTINT)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def tune(cfg="c4", reps=2, margin=0.02, device=0, log=print):
    mol = B.config_molecule(cfg)
    c = B.CONFIGS[cfg]
    g = MolGpu(mol, device, grad_tiles=None, eri_tiles=None)
    Cm = B.density_factor(g.nbf, c["rank"] or 40, c["seed"])
    D = torch.from_numpy(Cm @ Cm.T).to(f"cuda:{device}")
    t0 = time.time()
    g.grad_profile(True)
    _set_all(g, 0, 0)
    base, base_plan = _class_times(g, D, reps)
    log(f"planner: {sum(base.values()):.1f} ms over {len(base)} classes")
    runs = {}
    for tpq, order in CANDIDATES:
        _set_all(g, tpq, order)
        runs[(tpq, order)] = _class_times(g, D, reps)
        log(f"tpq {tpq} order {order}: {sum(runs[(tpq, order)][0].values()):.1f} ms")
    classes = pick(base, base_plan, runs, margin)
    # check: the table against the planner, profiled and in the normal launch
    _set_all(g, 0, 0)
    for key, t in classes.items():
        a, b = (int(x) for x in key.split(","))
        g.set_grad_tile(a, b, t["tpq"], t["order"])
    tuned, _ = _class_times(g, D, reps)
    ms_tuned = _gradient_ms(g, D, max(reps, 3))
    _set_all(g, 0, 0)
    ms_planner = _gradient_ms(g, D, max(reps, 3))
    table = {
        "workload": f"{cfg}: {mol.natom} atoms, {g.nbf} bf, Schwarz {CUTINT}; per-class kernel time, minimum of "
                    f"{reps} profiled gradients per candidate",
        "device": torch.cuda.get_device_name(device),
        "candidates": [list(x) for x in CANDIDATES],
        "margin": margin,
        "profiled_ms": {"planner": round(sum(base.values()), 2), "tuned": round(sum(tuned.values()), 2)},
        "gradient_ms": {"planner": round(ms_planner, 2), "tuned": round(ms_tuned, 2)},
        "tuning_seconds": round(time.time() - t0, 1),
        "classes": classes,
    }
    g.close()
    return table


def _eri_batch(g, sel, out, reps):
    """Per-class minimum kernel ms and plans over `reps` profiled batches."""
    g.eri_quartets(sel, out)
    torch.cuda.synchronize()
    best, plans = {}, {}
    for _ in range(reps):
        g.eri_quartets(sel, out)
        for k, (t, pl) in g.eri_class_times().items():
            if t < best.get(k, float("inf")):
                best[k], plans[k] = t, pl
    return best, plans


def _set_all_eri(g, tpq, order):
    for a in range(0, 8):
        for b in range(0, 8):
            g.set_eri_tile(a, b, tpq, order)


def _eri_ms(g, sel, out, reps):
    g.eri_profile(False)
    g.eri_quartets(sel, out)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.eri_quartets(sel, out)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def tune_eri(cfg="c2", sample=400_000, reps=2, margin=0.02, device=0, log=print):
    """ERI classes, timed on `sample` quartets drawn from the benchmark's seeded
    sample of the configuration; the table is checked on the whole sample."""
    mol = B.config_molecule(cfg)
    g = MolGpu(mol, device, eri_tiles=None)
    q = unique_quartets(len(mol.shells), g.schwarz(), CUTINT)
    full = q[np.sort(np.random.default_rng(0).choice(len(q), min(ERI_SAMPLE, len(q)), replace=False))]
    sel = full[np.sort(np.random.default_rng(1).choice(len(full), min(sample, len(full)), replace=False))]
    off = g.quartet_offsets(full)
    out = torch.empty(int(off[-1]), dtype=torch.float64, device=f"cuda:{device}")
    t0 = time.time()
    g.eri_profile(True)
    _set_all_eri(g, 0, 0)
    base, base_plan = _eri_batch(g, sel, out, reps)
    log(f"ERI planner: {sum(base.values()):.1f} ms over {len(base)} classes")
    runs = {}
    for tpq, order in ERI_CANDIDATES:
        _set_all_eri(g, tpq, order)
        runs[(tpq, order)] = _eri_batch(g, sel, out, reps)
        log(f"ERI tpq {tpq} order {order}: {sum(runs[(tpq, order)][0].values()):.1f} ms")
    classes = pick(base, base_plan, runs, margin)
    _set_all_eri(g, 0, 0)
    for key, t in classes.items():
        a, b = (int(x) for x in key.split(","))
        g.set_eri_tile(a, b, t["tpq"], t["order"])
    tuned, _ = _eri_batch(g, sel, out, reps)
    ms_tuned = _eri_ms(g, full, out, max(reps, 3))
    _set_all_eri(g, 0, 0)
    ms_planner = _eri_ms(g, full, out, max(reps, 3))
    table = {
        "workload": f"{cfg}: {mol.natom} atoms, {g.nbf} bf, Schwarz {CUTINT}; per-class kernel time on {len(sel)} "
                    f"quartets of the seeded {len(full)}-quartet sample, minimum of {reps} profiled batches",
        "device": torch.cuda.get_device_name(device),
        "candidates": [list(x) for x in ERI_CANDIDATES],
        "margin": margin,
        "profiled_ms": {"planner": round(sum(base.values()), 2), "tuned": round(sum(tuned.values()), 2)},
        "batch_ms": {"planner": round(ms_planner, 2), "tuned": round(ms_tuned, 2), "quartets": int(len(full))},
        "tuning_seconds": round(time.time() - t0, 1),
        "classes": classes,
    }
    del out
    g.close()
    return table


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--only", choices=("grad", "eri"), default=None)
    ap.add_argument("--cfg", default="c4")
    ap.add_argument("--eri-cfg", default="c2")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--margin", type=float, default=0.02)
    ap.add_argument("--out", default=GRAD_TILES)
    ap.add_argument("--eri-out", default=ERI_TILES)
    args = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    jobs = []
    if args.only in (None, "grad"):
        jobs.append((args.out, lambda: tune(args.cfg, args.reps, args.margin, log=log), "gradient_ms"))
    if args.only in (None, "eri"):
        jobs.append((args.eri_out, lambda: tune_eri(args.eri_cfg, reps=args.reps, margin=args.margin, log=log),
                     "batch_ms"))
    for path, run, key in jobs:
        table = run()
        with open(path, "w") as f:
            json.dump(table, f, indent=1)
            f.write("\n")
        print(json.dumps({k: table[k] for k in ("profiled_ms", key, "tuning_seconds")}
                         | {"classes_changed": len(table["classes"])}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
