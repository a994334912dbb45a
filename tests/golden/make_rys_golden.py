"""Generate tests/golden/rys_ref.npz from the reference's own Rys table.

Reads OpenMolcas's ``data/rysrw.ascii`` (layout of ``src/rys_util/
read_rysrw.F90:43-150``) and evaluates roots/weights exactly as
``src/rys_util/rys22.F90:36-47`` does for arguments below TMax:
``n = Map(int((T + 1.1 ddx)/ddx)); z = T - x0(n); R = sum_k Cff_k(n) z^k``.
Arguments are seeded uniform samples in [0, TMax(nRys)).

Run in a container that has the reference tree:
    python tests/golden/make_rys_golden.py /path/to/OpenMolcas
"""
from __future__ import annotations

import os
import sys

import numpy as np


def reference_tree():
    """The OpenMolcas source tree: the first argument, or $OPENMOLCAS_SRC."""
    src = os.environ.get("OPENMOLCAS_SRC")
    if not src:
        sys.exit("usage: python %s <OpenMolcas source tree>  (or set OPENMOLCAS_SRC)" % sys.argv[0])
    return src


def read_rysrw(path):
    with open(path) as f:
        lines = f.read().splitlines()
    start = None
    for k, ln in enumerate(lines):
        parts = ln.split()
        if len(parts) == 2 and all(p.lstrip("-").isdigit() for p in parts):
            start = k
            break
    toks = " ".join(lines[start:]).split()
    pos = 0

    def take(n, conv=float):
        nonlocal pos
        v = [conv(t.replace("D", "E").replace("d", "e")) for t in toks[pos:pos + n]]
        pos += n
        return v

    mrys, norder = take(2, int)
    acc = take(mrys)
    tmax = take(mrys)
    ddx = take(mrys)
    nmap = take(mrys, int)
    nx0 = take(mrys, int)
    maps, x0s = [], []
    for j in range(mrys):
        maps.append(np.array(take(nmap[j], int)))
        x0s.append(np.array(take(nx0[j])))
    ncff = 2 * (norder + 1)
    cffs = []
    for j in range(mrys):
        n = nx0[j] * (j + 1)
        cffs.append(np.array(take(n * ncff)).reshape(ncff, j + 1, nx0[j]))  # [coef][root][interval]
    return dict(mrys=mrys, norder=norder, acc=np.array(acc), tmax=np.array(tmax), ddx=np.array(ddx),
                maps=maps, x0s=x0s, cffs=cffs)


def eval_ref(tab, nrys, T):
    j = nrys - 1
    ddx = tab["ddx"][j]
    no = tab["norder"]
    dddx = ddx / 10.0 + ddx
    n = tab["maps"][j][int((T + dddx) / ddx) - 1] - 1
    z = T - tab["x0s"][j][n]
    c = tab["cffs"][j]
    roots = np.zeros(nrys)
    wts = np.zeros(nrys)
    for k in range(no, -1, -1):
        roots = roots * z + c[k, :, n]
        wts = wts * z + c[no + 1 + k, :, n]
    return roots, wts


def main(ref_root):
    tab = read_rysrw(os.path.join(ref_root, "data", "rysrw.ascii"))
    rng = np.random.default_rng(20240611)
    out = {}
    for nrys in range(1, tab["mrys"] + 1):
        tm = tab["tmax"][nrys - 1]
        T = np.concatenate([[0.0, 1e-8, 0.5, 1.0], rng.uniform(0.0, tm * 0.999, 60)])
        R = np.zeros((T.size, nrys))
        W = np.zeros((T.size, nrys))
        for k, t in enumerate(T):
            R[k], W[k] = eval_ref(tab, nrys, t)
        out[f"T{nrys}"] = T
        out[f"x{nrys}"] = R
        out[f"w{nrys}"] = W
    out["acc"] = tab["acc"]
    out["tmax"] = tab["tmax"]
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rys_ref.npz")
    np.savez(dst, **out)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
