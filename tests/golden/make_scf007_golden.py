"""Generate tests/golden/scf007_ch2_inline.npz from the reference's test 007.

The reference's ``test/standard/007.input`` runs singlet CH2 with an inline
basis (``C.cc-pvtz.dunning.10s5p2d.4s3p2d. / inline`` and
``H.cc-pvtz.dunning.5s2p.3s2p. / inline``: the basis data follow the label
inside the input), symmetry generators ``x y`` (C2v), conventional integrals
(``NoCD``) and a closed-shell SCF (``occupied 3 0 1 0``).  The checkfile holds
POTNUC (12 digits) and E_SCF (8 digits) of the first SCF.

An inline block is: ``charge lmax``, then per l (after optional ``*`` comment
lines) ``nprim ncontr``, the
exponents, the nprim x ncontr coefficients, then the centre lines (``name x y
z`` in bohr) up to ``end of basis``.  The unique centres are expanded by the
group of the generators (make_symgrad_golden.py).  Run in a container that has
the reference tree:
    python tests/golden/make_scf007_golden.py /path/to/OpenMolcas
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_scf071_golden import CHARGE  # noqa: E402
from make_symgrad_golden import group_ops  # noqa: E402


def reference_tree():
    """The OpenMolcas source tree: the first argument, or $OPENMOLCAS_SRC."""
    src = os.environ.get("OPENMOLCAS_SRC")
    if not src:
        sys.exit("usage: python %s <OpenMolcas source tree>  (or set OPENMOLCAS_SRC)" % sys.argv[0])
    return src


def numbers(lines, k, n):
    vals = []
    while len(vals) < n:
        if not lines[k].lstrip().startswith("*"):
            vals.extend(float(v) for v in lines[k].split())
        k += 1
    return np.array(vals[:n]), k


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    gens, blocks = [], []  # blocks: (element, charge, shells, centres)
    k = 0
    while k < len(lines):
        ln = lines[k].strip().lower()
        if ln == "end of input" and blocks:
            break  # first &SEWARD only
        if ln == "symmetry":
            gens = lines[k + 1].split()
            k += 2
            continue
        if ln == "basis set":
            label = lines[k + 1].strip()
            assert label.lower().endswith("/ inline"), label
            el = label.split(".")[0]
            charge, lmax = lines[k + 2].split()
            k += 3
            shells = []
            for l in range(int(lmax) + 1):
                while lines[k].lstrip().startswith("*"):
                    k += 1
                npr, nco = (int(v) for v in lines[k].split())
                exps, k = numbers(lines, k + 1, npr)
                coef, k = numbers(lines, k, npr * nco)
                shells.append((l, exps, coef.reshape(npr, nco)))
            centres = []
            while lines[k].strip().lower() != "end of basis":
                t = lines[k].split()
                assert len(t) == 4, lines[k]  # bohr
                centres.append([float(v) for v in t[1:4]])
                k += 1
            blocks.append((el, float(charge), shells, centres))
        k += 1
    chk = {}
    for ln in lines:
        m = re.match(r'#> (\w+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return gens, blocks, chk


def main(ref):
    gens, blocks, chk = read_input(os.path.join(ref, "test", "standard", "007.input"))
    ops = group_ops(gens)
    xyz, q = [], []
    sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], []
    for el, charge, shells, centres in blocks:
        assert CHARGE[el.upper()] == charge
        for r in centres:
            r = np.array(r)
            first = len(xyz)
            for o in ops:
                img = r * np.array(o)
                if all(np.linalg.norm(img - np.array(x)) > 1e-8 for x in xyz[first:]):
                    xyz.append(img.tolist())
                    q.append(charge)
                    for l, e, c in shells:
                        sh_atom.append(len(xyz) - 1)
                        sh_l.append(l)
                        sh_np.append(len(e))
                        sh_nc.append(c.shape[1])
                        exps.append(e)
                        coefs.append(c.reshape(-1))
    out = dict(coords=np.array(xyz), charges=np.array(q), generators=np.array(" ".join(gens)),
               shell_atom=np.array(sh_atom, np.int32), shell_l=np.array(sh_l, np.int32),
               shell_nprim=np.array(sh_np, np.int32), shell_ncontr=np.array(sh_nc, np.int32),
               exps=np.concatenate(exps), coefs=np.concatenate(coefs))
    for key in ("POTNUC", "E_SCF"):
        out[key] = np.array(chk[key][0])
        out[key + "_digits"] = np.array(chk[key][1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scf007_ch2_inline.npz")
    np.savez(dst, **out)
    print(dst, len(xyz), "atoms", sh_l, sh_np, sh_nc, float(out["E_SCF"]))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
