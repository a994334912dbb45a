"""Generate tests/golden/scf065_co_ccpvdz.npz from the reference's test 065.

The reference's ``test/standard/065.input`` runs CO in cc-pVDZ with no
symmetry and a full Cholesky decomposition of the ERIs (``&SEWARD
Cholesky``, default ThrCom 1e-4), then ``&SCF`` from the orbitals embedded in
the input with ``Occupied = 7`` and ``Frozen = 7``: every occupied orbital is
frozen (``scf/aufbau.F90:68`` optimises only nOrb - nFro), so the checked
``E_SCF`` is the RHF energy of the embedded orbitals.  Its checkfile also holds
``POTNUC`` and the first packed element of the kinetic and nuclear-attraction
matrices (``SEWARD_KINETIC``/``SEWARD_ATTRACT``, ``integral_util/oneel.F90:302-303``).

This script reads, from a reference tree:
  * the geometry (bohr), the basis label and the embedded orbital file
    (``#ORB`` coefficients and ``#OCC`` occupations, INPORB 1.0 layout:
    4 numbers of 18 characters per line) from ``test/standard/065.input``;
  * the C and O entries of ``basis_library/CC-PVDZ`` (per atom: charge and
    lmax, then per l ``nprim ncontr``, the exponents, the nprim x ncontr
    coefficient matrix; un-normalised, as the library stores them);
and writes the arrays the tests need.  Run in a container that has the
reference tree:
    python tests/golden/make_scf065_golden.py /path/to/OpenMolcas
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
    # geometry block of &GATEWAY: "Coord = n", "Bohr", n lines "El x y z"
    k = next(i for i, ln in enumerate(lines) if re.match(r"\s*Coord\s*=", ln, re.I))
    nat = int(lines[k].split("=")[1])
    assert lines[k + 1].strip().lower() == "bohr"
    elems, xyz = [], []
    for ln in lines[k + 2:k + 2 + nat]:
        t = ln.split()
        elems.append(t[0])
        xyz.append([float(v) for v in t[1:4]])
    basis = next(ln.split("=")[1].strip() for ln in lines if re.match(r"\s*Basis\s*=", ln, re.I))
    # the embedded orbital file
    i0 = next(i for i, ln in enumerate(lines) if ln.strip() == "#ORB")
    i1 = next(i for i, ln in enumerate(lines) if ln.strip() == "#OCC")
    i2 = next(i for i, ln in enumerate(lines) if ln.strip() == "#ONE")

    def numbers(block):
        vals = []
        for ln in block:
            if ln.startswith("*") or ln.startswith("#"):
                continue
            for p in range(0, len(ln), 18):
                s = ln[p:p + 18].strip()
                if s:
                    vals.append(float(s))
        return vals

    orb = []
    cur = None
    for ln in lines[i0 + 1:i1]:
        if ln.startswith("* ORBITAL"):
            cur = []
            orb.append(cur)
        else:
            cur.extend(numbers([ln]))
    occ = numbers(lines[i1 + 1:i2])
    # check values: the third checkfile section (after &SCF)
    chk = {}
    for ln in lines:
        m = re.match(r'#> (\w+)="([-0-9.eE+]+)"/(\d+)', ln)
        if m and m.group(1) not in chk:
            chk[m.group(1)] = (float(m.group(2)), int(m.group(3)))
    return elems, np.array(xyz), basis, np.array(orb), np.array(occ), chk


def read_library(path, elem):
    with open(path) as f:
        lines = f.read().splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.upper().startswith("/" + elem.upper() + ".CC-PVDZ.DUNNING"))
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


def main(ref):
    elems, xyz, basis, orb, occ, chk = read_input(os.path.join(ref, "test", "standard", "065.input"))
    assert basis.lower() == "cc-pvdz", basis
    lib = os.path.join(ref, "basis_library", "CC-PVDZ")
    out = dict(coords=xyz, orbitals=orb, occupation=occ)
    charges, sh_atom, sh_l, sh_np, sh_nc, exps, coefs = [], [], [], [], [], [], []
    for a, el in enumerate(elems):
        q, shells = read_library(lib, el)
        charges.append(q)
        for l, e, c in shells:
            sh_atom.append(a)
            sh_l.append(l)
            sh_np.append(len(e))
            sh_nc.append(c.shape[1])
            exps.append(e)
            coefs.append(c.reshape(-1))  # row-major [nprim, ncontr]
    out.update(charges=np.array(charges), shell_atom=np.array(sh_atom, np.int32), shell_l=np.array(sh_l, np.int32),
               shell_nprim=np.array(sh_np, np.int32), shell_ncontr=np.array(sh_nc, np.int32),
               exps=np.concatenate(exps), coefs=np.concatenate(coefs))
    for key in ("POTNUC", "SEWARD_KINETIC", "SEWARD_ATTRACT", "SCF_ITER", "E_SCF"):
        out[key] = np.array(chk[key][0])
        out[key + "_digits"] = np.array(chk[key][1])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scf065_co_ccpvdz.npz")
    np.savez(dst, **out)
    print(dst, {k: out[k] for k in ("POTNUC", "SEWARD_KINETIC", "SEWARD_ATTRACT", "E_SCF")}, orb.shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else reference_tree())
