"""Generate a gradient fixture from one of the reference's SCF + Alaska tests
that use point-group symmetry (tests/golden/grad020_ch4_ccpvdz.npz from test
020, tests/golden/grad023_ch2o2_ccpvdz.npz from test 023, and tests 019, 021
and 049 likewise).

Test 020 optimises CH4 in cc-pVDZ with the symmetry generators ``x z`` (C2v),
test 023 a CH2O2 transition state in cc-pVDZ with the generator ``Y`` (Cs);
both use conventional integrals (``NoCD``): ``&SEWARD``, ``&SCF``,
``&ALASKA``.  Their checkfiles hold, for the first geometry, POTNUC, E_SCF
(8 digits) and GRAD (6 digits).  With symmetry, GRAD
lists the symmetry-allowed Cartesian components of the symmetry-unique
centres: centre by centre in input order, x, y, z, keeping a component when
no operation that leaves the centre in place changes its sign.

This script reads, from a reference tree:
  * the generators after ``Symmetry`` and the ``Basis Set`` blocks of
    ``&SEWARD`` (label line, then ``name x y z`` in bohr; lines starting with
    ``*`` are comments) from ``test/standard/<id>.input``, and the first
    POTNUC, E_SCF and GRAD entries of its checkfile;
  * the entries of ``basis_library/CC-PVDZ`` for its elements (the reader of
    make_grad862_golden.py);
expands every unique centre by the group the generators span (a generator
names the coordinates whose sign it changes), and writes the molecule, the
index of each atom's unique centre, and for every GRAD entry the atom and
component it belongs to.  Run in a container that has the reference tree:
    python tests/golden/make_symgrad_golden.py /path/to/OpenMolcas 020 grad020_ch4_ccpvdz
    python tests/golden/make_symgrad_golden.py /path/to/OpenMolcas 023 grad023_ch2o2_ccpvdz
    python tests/golden/make_symgrad_golden.py /path/to/OpenMolcas 019 grad019_c4h8_sto3g
    python tests/golden/make_symgrad_golden.py /path/to/OpenMolcas 021 grad021_c6h6_sto3g
    python tests/golden/make_symgrad_golden.py /path/to/OpenMolcas 049 grad049_ch2o2_ccpvdz
"""
from __future__ import annotations

import itertools
import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_grad862_golden import read_library  # noqa: E402

CHARGE = {"H": 1.0, "C": 6.0, "N": 7.0, "O": 8.0}


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    gens, centres = [], []  # centres: (element, basis label, xyz bohr)
    k = 0
    while k < len(lines):
        ln = lines[k].strip()
        if ln.lower() == "symmetry":
            gens = lines[k + 1].split()
            k += 2
            continue
        if ln.lower() == "basis set":
            k += 1
            while lines[k].lstrip().startswith("*"):
                k += 1
            label = lines[k].strip()
            el, bas = label.split(".")[0], label.split(".")[1]
            k += 1
            while lines[k].strip().lower() != "end of basis":
                if not lines[k].lstrip().startswith("*"):
                    t = lines[k].split()
                    assert len(t) == 4, lines[k]  # bohr
                    centres.append((el, bas, [float(v) for v in t[1:4]]))
                k += 1
        k += 1
    chk = {}
    for ln in lines:
        m = re.match(r'#> ([\w\[\]]+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return gens, centres, chk


def group_ops(gens):
    """Sign vectors of every element of the group the generators span."""
    ops = {(1, 1, 1)}
    for g in gens:
        s = tuple(-1 if c in g.lower() else 1 for c in "xyz")
        ops |= {tuple(a * b for a, b in zip(o, s)) for o in ops}
    changed = True
    while changed:
        new = {tuple(a * b for a, b in zip(o1, o2)) for o1, o2 in itertools.product(ops, ops)}
        changed = not new <= ops
        ops |= new
    return sorted(ops, reverse=True)


def main(ref, test_id, name):
    gens, centres, chk = read_input(os.path.join(ref, "test", "standard", test_id + ".input"))
    ops = group_ops(gens)
    xyz, unique_of, elems, labels = [], [], [], []
    comps = []  # (atom index, component) per GRAD entry
    for u, (el, bas, r) in enumerate(centres):
        r = np.array(r)
        first = len(xyz)
        for o in ops:
            img = r * np.array(o)
            if all(np.linalg.norm(img - np.array(x)) > 1e-8 for x in xyz[first:]):
                xyz.append(img.tolist())
                unique_of.append(u)
                elems.append(el)
                labels.append(bas)
        stab = [o for o in ops if np.linalg.norm(r * np.array(o) - r) < 1e-8]
        for c in range(3):
            if all(o[c] == 1 for o in stab):
                comps.append((first, c))
    xyz = np.array(xyz)
    q = np.array([CHARGE[e.upper()] for e in elems])
    out = dict(coords=xyz, charges=q, unique_of=np.array(unique_of, np.int32),
               grad_atom=np.array([a for a, _ in comps], np.int32), grad_comp=np.array([c for _, c in comps], np.int32),
               generators=np.array(" ".join(gens)))
    sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], []
    for ia, (el, bas) in enumerate(zip(elems, labels)):
        qq, shells = read_library(os.path.join(ref, "basis_library", bas.upper()), el, bas)
        assert qq == q[ia]
        for l, e, c in shells:
            sh_atom.append(ia)
            sh_l.append(l)
            sh_np.append(len(e))
            sh_nc.append(c.shape[1])
            exps.append(e)
            coefs.append(c.reshape(-1))
    out.update(shell_atom=np.array(sh_atom, np.int32), shell_l=np.array(sh_l, np.int32),
               shell_nprim=np.array(sh_np, np.int32), shell_ncontr=np.array(sh_nc, np.int32),
               exps=np.concatenate(exps), coefs=np.concatenate(coefs))
    for key in ("POTNUC", "E_SCF"):
        out[key] = np.array(chk[key][0])
        out[key + "_digits"] = np.array(chk[key][1])
    out["GRAD"] = np.array([chk[f"GRAD[{i}]"][0] for i in range(len(comps))])
    out["GRAD_digits"] = np.array(chk["GRAD[0]"][1])
    assert f"GRAD[{len(comps)}]" not in chk
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), name + ".npz")
    np.savez(dst, **out)
    print(dst, len(xyz), "atoms", comps, float(out["E_SCF"]), out["GRAD"].tolist())


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], sys.argv[3])
