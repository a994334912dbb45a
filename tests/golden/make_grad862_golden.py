"""Generate tests/golden/grad862_h2o_631g.npz from the reference's test 862.

The reference's ``test/standard/862.input`` optimises water in 6-31G with no
symmetry and conventional (non-Cholesky) integrals: ``&SEWARD``, ``&SCF``,
``&ALASKA`` in a loop.  Its checkfile holds, for the first geometry, the
converged ``E_SCF`` (8 digits) and the nuclear gradient ``GRAD[0..8]``
(6 digits, atom-major x, y, z), plus the first packed kinetic and attraction
integrals (``integral_util/oneel.F90:302-303``).

This script reads, from a reference tree:
  * the first geometry (an XYZ block in angstrom after ``Coord``) and the
    basis label from ``test/standard/862.input``, and the check values of the
    first geometry (the first occurrence of each label);
  * the O and H entries of ``basis_library/6-31G`` (charge and lmax, then per
    l ``nprim ncontr``, exponents, the nprim x ncontr coefficient matrix);
  * the Bohr radius of the default CODATA set from
    ``src/system_util/constants.F90`` (angstrom -> bohr);
and writes the arrays the tests need.  Run in a container that has the
reference tree:
    python tests/golden/make_grad862_golden.py /path/to/OpenMolcas
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np


def reference_tree():
    """The OpenMolcas source tree: the first argument, or $OPENMOLCAS_SRC."""
    src = os.environ.get("OPENMOLCAS_SRC")
    if not src:
        sys.exit("usage: python %s <OpenMolcas source tree>  (or set OPENMOLCAS_SRC)" % sys.argv[0])
    return src


def read_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.strip().lower() == "coord")
    nat = int(lines[k + 1].split()[0])
    elems, xyz = [], []
    for ln in lines[k + 3:k + 3 + nat]:
        t = ln.split()
        elems.append(t[0])
        xyz.append([float(v) for v in t[1:4]])
    basis = next(ln.split("=")[1].strip() for ln in lines if re.match(r"\s*Basis\s*=", ln, re.I))
    chk = {}
    for ln in lines:
        m = re.match(r'#> ([\w\[\]]+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return elems, np.array(xyz), basis, chk


def read_library(path, elem, label):
    with open(path) as f:
        lines = f.read().splitlines()
    head = "/" + elem.upper() + "." + label.upper() + "."
    k = next(i for i, ln in enumerate(lines) if ln.upper().startswith(head))
    k += 3  # header, reference, comment
    charge, lmax = lines[k].split()
    charge, lmax = float(charge), int(lmax)
    k += 1
    shells = []
    for l in range(lmax + 1):
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
        shells.append((l, exps, np.array(coef).reshape(npr, nco)))
    return charge, shells


def bohr_radius_angstrom(path):
    src = open(path).read()
    cset = re.search(r"#define CODATA_SET (\d+)", src).group(1)
    block = src.split("#if CODATA_SET == " + cset, 1)[1] if ("#if CODATA_SET == " + cset) in src else \
        src.split("#elif CODATA_SET == " + cset, 1)[1]
    val = re.search(r"CONST_BOHR_RADIUS_IN_SI_\s+([0-9.eE+-]+)_wp", block).group(1)
    return float(val) * 1e10, int(cset)


def main(ref):
    elems, xyz_ang, basis, chk = read_input(os.path.join(ref, "test", "standard", "862.input"))
    a0, cset = bohr_radius_angstrom(os.path.join(ref, "src", "system_util", "constants.F90"))
    lib = os.path.join(ref, "basis_library", basis.upper())
    out = dict(coords=xyz_ang / a0, coords_angstrom=xyz_ang, bohr_radius_angstrom=np.array(a0),
               codata_set=np.array(cset))
    charges, sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], [], []
    for a, el in enumerate(elems):
        q, shells = read_library(lib, el, basis)
        charges.append(q)
        for l, e, c in shells:
            sh_atom.append(a)
            sh_l.append(l)
            sh_np.append(len(e))
            sh_nc.append(c.shape[1])
            exps.append(e)
            coefs.append(c.reshape(-1))
    out.update(charges=np.array(charges), shell_atom=np.array(sh_atom, np.int32), shell_l=np.array(sh_l, np.int32),
               shell_nprim=np.array(sh_np, np.int32), shell_ncontr=np.array(sh_nc, np.int32),
               exps=np.concatenate(exps), coefs=np.concatenate(coefs))
    for key in ("SEWARD_KINETIC", "SEWARD_ATTRACT", "SCF_ITER", "E_SCF"):
        out[key] = np.array(chk[key][0])
        out[key + "_digits"] = np.array(chk[key][1])
    out["GRAD"] = np.array([chk[f"GRAD[{i}]"][0] for i in range(3 * len(elems))]).reshape(-1, 3)
    out["GRAD_digits"] = np.array(chk["GRAD[0]"][1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grad862_h2o_631g.npz")
    np.savez(dst, **out)
    print(dst, float(out["E_SCF"]), out["GRAD"].tolist(), a0, cset)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
