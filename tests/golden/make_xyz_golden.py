"""Generate a fixture from one of the reference's no-symmetry tests whose
&GATEWAY gives the geometry as an XYZ block in angstrom and one basis label
for every atom: tests 078 (water dimer, 6-31G), 090 (STO-3G), 094 and 095
(HCN/CNH, STO-3G), and 099 (1,2-dioxetanone, 6-31G), whose &SCF starts from
an orbital file the input embeds (``FILE = name``: INPORB, ``#ORB`` vectors
and ``#OCC`` occupations, stored as ``orbitals`` and ``occupation``).  GRAD,
when the checkfile has one and the test checks it, is its first gradient:
the SCF gradient of the first geometry for 094 (&SCF then &SLAPAF), an MP2
gradient for 078 and 090 (&MBPT2 before &SLAPAF).

The XYZ block is either inline (``Coord = N`` followed by N atom lines, or
``Coord`` followed by the count line, a title line and the atoms) or a file
the input embeds (``Coord = name.xyz`` with a ``>> FILE name.xyz`` block,
ended by the next ``>> FILE`` or ``>> EOF``: count, title, atoms).  The script reads the first such
geometry, the ``Basis =`` label, the matching entries of the basis library
(the reader of make_grad862_golden.py), the Bohr radius of the CODATA set that
reproduces POTNUC (make_scf071_golden.py), and the first POTNUC, E_SCF and,
when present, GRAD of the checkfile.  Run in a container that has the
reference tree:
    python tests/golden/make_xyz_golden.py /path/to/OpenMolcas 094 scf094_hcn_sto3g
(and 078 scf078_h2o2_631g, 090 scf090_sto3g, 095 scf095_hcn_sto3g,
099 scf099_c2h2o3_631g).
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_grad862_golden import read_library  # noqa: E402
from make_scf071_golden import CHARGE, bohr_radii  # noqa: E402


def atom_lines(lines, n):
    els, xyz = [], []
    for ln in lines[:n]:
        t = ln.split()
        els.append(re.match(r"[A-Za-z]+", t[0]).group(0).capitalize())
        xyz.append([float(v) for v in t[1:4]])
    return els, xyz


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    files = {}
    for k, ln in enumerate(lines):
        m = re.match(r"\s*>>>?\s*FILE\s+(\S+)", ln, re.I)
        if m:
            end = next(j for j in range(k + 1, len(lines)) if re.match(r"\s*>>>?\s*(EOF|FILE)", lines[j], re.I))
            files[m.group(1)] = lines[k + 1:end]
    geo = None
    for k, ln in enumerate(lines):
        m = re.match(r"\s*coord\s*(=\s*(\S+))?\s*$", ln, re.I)
        if not m:
            continue
        arg = m.group(2)
        if arg is None:  # count line, title, atoms
            n = int(lines[k + 1].split()[0])
            geo = atom_lines(lines[k + 3:], n)
        elif arg.isdigit():  # N atom lines (a title line may precede them)
            n = int(arg)
            body = [x for x in lines[k + 1:k + 2 + n] if x.strip()]
            if len(body[0].split()) < 4:
                body = body[1:]
            geo = atom_lines(body, n)
        else:  # embedded file
            body = files[arg]
            n = int(body[0].split()[0])
            geo = atom_lines(body[2:], n)
        break
    basis = next(re.split(r"=", ln, 1)[1].strip() for ln in lines if re.match(r"\s*basis\s*=", ln, re.I))
    orbs = None
    for ln in lines:
        m = re.match(r"\s*file\s*=\s*(\S+)", ln, re.I)
        if m and m.group(1) in files and files[m.group(1)][0].startswith("#INPORB"):
            orbs = read_inporb(files[m.group(1)])
    chk = {}
    for ln in lines:
        m = re.match(r'#> ([\w\[\]]+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    nocheck = any(re.search(r"MOLCAS_NOCHECK=.*GRAD", ln) for ln in lines)
    return geo, basis, chk, orbs, nocheck


def read_inporb(body):
    """(orbitals [norb, nbf], occupations) of an INPORB 2.x file, one symmetry."""
    i0 = body.index("#ORB")
    i1 = next(i for i, ln in enumerate(body) if ln.startswith("#OCC"))
    i2 = next(i for i, ln in enumerate(body) if i > i1 and ln.startswith("#") and not ln.startswith("#OCC"))
    orbs, cur = [], None
    for ln in body[i0 + 1:i1]:
        if ln.startswith("* ORBITAL"):
            cur = []
            orbs.append(cur)
        elif not ln.startswith("*"):
            cur.extend(float(v) for v in ln.split())
    occ = [float(v) for ln in body[i1 + 1:i2] if not ln.startswith("*") for v in ln.split()]
    return np.array(orbs), np.array(occ)


def main(ref, test_id, name):
    (els, xyz), basis, chk, orbs, nocheck = read_input(os.path.join(ref, "test", "standard", test_id + ".input"))
    xyz = np.array(xyz)
    q = np.array([CHARGE[e.upper()] for e in els])
    best = None
    for cset, a0 in sorted(bohr_radii(os.path.join(ref, "src", "system_util", "constants.F90")).items()):
        R = xyz / a0
        e = sum(q[i] * q[j] / np.linalg.norm(R[i] - R[j]) for i in range(len(q)) for j in range(i))
        d = abs(e - chk["POTNUC"][0])
        if best is None or d < best[0]:
            best = (d, cset, a0)
    _, cset, a0 = best
    out = dict(coords=xyz / a0, coords_angstrom=xyz, charges=q, bohr_radius_angstrom=np.array(a0),
               codata_set=np.array(cset))
    lib = os.path.join(ref, "basis_library", basis.upper())
    sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], []
    for ia, el in enumerate(els):
        qq, shells = read_library(lib, el, basis)
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
    if orbs is not None:
        out["orbitals"], out["occupation"] = orbs
    if "GRAD[0]" in chk and not nocheck:
        out["GRAD"] = np.array([chk[f"GRAD[{i}]"][0] for i in range(3 * len(els))]).reshape(-1, 3)
        out["GRAD_digits"] = np.array(chk["GRAD[0]"][1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), name + ".npz")
    np.savez(dst, **out)
    print(dst, len(els), "atoms", basis, float(out["E_SCF"]), "GRAD" in out, "CODATA", cset, "POTNUC residual",
          best[0])


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], sys.argv[3])
