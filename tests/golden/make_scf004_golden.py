"""Generate tests/golden/scf004_h2o_anos.npz from the reference's test 004.

The reference's ``test/standard/004.input`` runs water in ANO-S with the
contractions ``H.ano-s...2s1p.`` and ``O.ano-s...3s2p1d.``, symmetry
generators ``x y`` (C2v), conventional integrals (``NoCD``) and a closed-shell
SCF.  ANO contractions are general: every primitive of a shell enters every
contracted function.  The checkfile holds POTNUC (12 digits) and E_SCF
(8 digits) of the first SCF.

This script reads, from a reference tree:
  * the generators after ``Symmetry`` and the ``Basis set`` blocks of the
    first ``&SEWARD`` (label line, then ``name x y z Angstrom``) from
    ``test/standard/004.input``, and its first POTNUC and E_SCF;
  * the H and O entries of ``basis_library/ANO-S``: after the header, the
    reference and ``*`` comment lines and an optional ``Options`` ...
    ``EndOptions`` block, the charge and lmax line, then per l ``nprim
    ncontr``, the exponents, the nprim x ncontr coefficients and, with the
    ``OrbitalEnergies`` option, a count n and n orbital energies (with
    ``FockOperator``, n and an n x n matrix); the
    label's ``3s2p1d`` keeps the first 3 s, 2 p and 1 d columns and drops
    higher l;
  * the Bohr radius of the CODATA set that reproduces POTNUC
    (make_scf071_golden.py);
expands the symmetry-unique centres by the group of the generators
(make_symgrad_golden.py) and writes the molecule and the check values.
Run in a container that has the reference tree:
    python tests/golden/make_scf004_golden.py /path/to/OpenMolcas
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_scf071_golden import CHARGE, bohr_radii  # noqa: E402
from make_symgrad_golden import group_ops  # noqa: E402


def reference_tree():
    """The OpenMolcas source tree: the first argument, or $OPENMOLCAS_SRC."""
    src = os.environ.get("OPENMOLCAS_SRC")
    if not src:
        sys.exit("usage: python %s <OpenMolcas source tree>  (or set OPENMOLCAS_SRC)" % sys.argv[0])
    return src


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    gens, centres = [], []
    k = 0
    while k < len(lines):
        ln = lines[k].strip()
        if ln.lower().startswith("&seward") and centres:
            break  # first &SEWARD only
        if ln.lower() == "symmetry":
            gens = lines[k + 1].split()
            k += 2
            continue
        if ln.lower() == "basis set":
            label = lines[k + 1].strip()
            k += 2
            while lines[k].strip().lower() != "end of basis":
                t = lines[k].split()
                assert t[4].lower().startswith("angstrom"), lines[k]
                centres.append((label, [float(v) for v in t[1:4]]))
                k += 1
        k += 1
    chk = {}
    for ln in lines:
        m = re.match(r'#> (\w+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return gens, centres, chk


def read_ano(path, elem, family, keep):
    """Shells (l, exps, coef[nprim, ncontr]) keeping keep[l] columns."""
    with open(path) as f:
        lines = f.read().splitlines()
    head = "/" + elem.upper() + "." + family.upper() + "."
    k = next(i for i, ln in enumerate(lines) if ln.upper().startswith(head)) + 2
    orb_energies = fock = False
    while not re.match(r"^\s*\d+\.\d*\s+\d+\s*$", lines[k]):
        if lines[k].strip().lower() == "options":
            k += 1
            while lines[k].strip().lower() != "endoptions":
                opt = lines[k].strip().lower()
                assert not opt.startswith("cartesian"), opt
                orb_energies |= opt.startswith("orbitalenergies")
                fock |= opt.startswith("fockoperator")
                k += 1
        k += 1
    charge, lmax = lines[k].split()
    k += 1
    shells = []
    for l in range(int(lmax) + 1):
        while lines[k].lstrip().startswith("*"):
            k += 1
        npr, nco = (int(v) for v in lines[k].split())
        k += 1
        exps = np.array([float(lines[k + i].split()[0]) for i in range(npr)])
        k += npr
        coef = []
        while len(coef) < npr * nco:
            coef.extend(float(v) for v in lines[k].split())
            k += 1
        if orb_energies or fock:  # n, then n orbital energies or an n x n Fock matrix
            ne = int(lines[k].split()[0])
            ne = ne * ne if fock else ne
            k += 1
            got = 0
            while got < ne:
                got += len(lines[k].split())
                k += 1
        if l < len(keep) and keep[l] > 0:
            c = np.array(coef).reshape(npr, nco)[:, : keep[l]]
            shells.append((l, exps, c))
    return float(charge), shells


def main(ref):
    gens, centres, chk = read_input(os.path.join(ref, "test", "standard", "004.input"))
    ops = group_ops(gens)
    atoms = []  # (label, xyz angstrom)
    for label, r in centres:
        r = np.array(r)
        first = len(atoms)
        for o in ops:
            img = r * np.array(o)
            if all(np.linalg.norm(img - np.array(x[1])) > 1e-8 for x in atoms[first:]):
                atoms.append((label, img.tolist()))
    xyz = np.array([a[1] for a in atoms])
    q = np.array([CHARGE[a[0].split(".")[0].upper()] for a in atoms])
    best = None
    for cset, a0 in sorted(bohr_radii(os.path.join(ref, "src", "system_util", "constants.F90")).items()):
        R = xyz / a0
        e = sum(q[i] * q[j] / np.linalg.norm(R[i] - R[j]) for i in range(len(q)) for j in range(i))
        d = abs(e - chk["POTNUC"][0])
        if best is None or d < best[0]:
            best = (d, cset, a0)
    _, cset, a0 = best
    out = dict(coords=xyz / a0, coords_angstrom=xyz, charges=q, bohr_radius_angstrom=np.array(a0),
               codata_set=np.array(cset), generators=np.array(" ".join(gens)))
    sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], []
    for ia, (label, _) in enumerate(atoms):
        parts = label.split(".")
        el, family, contr = parts[0], parts[1], parts[4]
        keep = [int(n) for n in re.findall(r"(\d+)[spdfg]", contr.lower())]
        letters = re.findall(r"\d+([spdfg])", contr.lower())
        assert letters == list("spdfg"[: len(letters)]), contr
        qq, shells = read_ano(os.path.join(ref, "basis_library", family.upper()), el, family, keep)
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
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scf004_h2o_anos.npz")
    np.savez(dst, **out)
    print(dst, len(atoms), "atoms", sh_l, sh_np, sh_nc, float(out["E_SCF"]), "CODATA", cset, "POTNUC residual",
          best[0])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
