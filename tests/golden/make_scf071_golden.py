"""Generate tests/golden/scf071_h2o_ccpvtz.npz from the reference's test 071.

The reference's ``test/standard/071.input`` runs water in cc-pVTZ (s to f
shells, all real spherical) with no symmetry and conventional integrals
(``NoCD``), then a closed-shell SCF (``Occupied 5``).  Its checkfile holds
POTNUC (12 digits) and, first, the converged E_SCF (8 digits).

This script reads, from a reference tree:
  * the ``Basis set`` blocks of ``&SEWARD`` (a label line such as
    ``H.cc-pvtz....``, then ``name x y z Angstrom`` lines) from
    ``test/standard/071.input`` and the first POTNUC and E_SCF of its checkfile;
  * the H and O entries of ``basis_library/CC-PVTZ`` (the reader of
    make_grad862_golden.py);
  * the Bohr radii of every CODATA set in ``src/system_util/constants.F90``,
    keeping the one whose nuclear repulsion reproduces POTNUC best (the
    checkfile predates the current default set);
and writes the arrays the tests need.  Run in a container that has the
reference tree:
    python tests/golden/make_scf071_golden.py /path/to/OpenMolcas
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_grad862_golden import read_library  # noqa: E402

CHARGE = {"H": 1.0, "C": 6.0, "N": 7.0, "O": 8.0}


def reference_tree():
    """The OpenMolcas source tree: the first argument, or $OPENMOLCAS_SRC."""
    src = os.environ.get("OPENMOLCAS_SRC")
    if not src:
        sys.exit("usage: python %s <OpenMolcas source tree>  (or set OPENMOLCAS_SRC)" % sys.argv[0])
    return src


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    atoms = []  # (element, label, xyz angstrom)
    k = 0
    while k < len(lines):
        if lines[k].strip().lower() == "basis set":
            label = lines[k + 1].strip()
            el, bas = label.split(".")[0], label.split(".")[1]
            k += 2
            while lines[k].strip().lower() != "end of basis":
                t = lines[k].split()
                assert t[4].lower().startswith("angstrom"), lines[k]
                atoms.append((el, bas, [float(v) for v in t[1:4]]))
                k += 1
        k += 1
    chk = {}
    for ln in lines:
        m = re.match(r'#> (\w+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return atoms, chk


def bohr_radii(path):
    src = open(path).read()
    return {int(s): float(v) * 1e10 for s, v in
            re.findall(r"CODATA_SET == (\d+)\s*\n(?:#.*\n)*?#\s*define CONST_BOHR_RADIUS_IN_SI_\s+([0-9.eE+-]+)_wp",
                       src)}


def main(ref):
    atoms, chk = read_input(os.path.join(ref, "test", "standard", "071.input"))
    xyz = np.array([a[2] for a in atoms])
    q = np.array([CHARGE[a[0].upper()] for a in atoms])
    best = None
    for cset, a0 in sorted(bohr_radii(os.path.join(ref, "src", "system_util", "constants.F90")).items()):
        R = xyz / a0
        e = sum(q[i] * q[j] / np.linalg.norm(R[i] - R[j]) for i in range(len(q)) for j in range(i))
        d = abs(e - chk["POTNUC"][0])
        if best is None or d < best[0]:
            best = (d, cset, a0)
    _, cset, a0 = best
    out = dict(coords=xyz / a0, coords_angstrom=xyz, bohr_radius_angstrom=np.array(a0), codata_set=np.array(cset))
    sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], []
    for ia, (el, bas, _) in enumerate(atoms):
        qq, shells = read_library(os.path.join(ref, "basis_library", bas.upper()), el, bas)
        assert qq == q[ia]
        for l, e, c in shells:
            sh_atom.append(ia)
            sh_l.append(l)
            sh_np.append(len(e))
            sh_nc.append(c.shape[1])
            exps.append(e)
            coefs.append(c.reshape(-1))
    out.update(charges=q, shell_atom=np.array(sh_atom, np.int32), shell_l=np.array(sh_l, np.int32),
               shell_nprim=np.array(sh_np, np.int32), shell_ncontr=np.array(sh_nc, np.int32),
               exps=np.concatenate(exps), coefs=np.concatenate(coefs))
    for key in ("POTNUC", "E_SCF"):
        out[key] = np.array(chk[key][0])
        out[key + "_digits"] = np.array(chk[key][1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scf071_h2o_ccpvtz.npz")
    np.savez(dst, **out)
    print(dst, float(out["E_SCF"]), "CODATA", cset, "POTNUC residual", best[0])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
