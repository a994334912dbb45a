"""Seeded synthetic molecules and basis sets for the two-electron path.

Basis conventions follow the reference (OpenMolcas):

* shells are (atom, l) with *general* contraction: ``coef[nprim, ncontr]``
  (``integral_util/twoel_nosym.F90:96-99``, ``Shells(:)%pCff``);
* contraction coefficients are normalised exactly like ``Nrmlz``
  (``gateway_util/nrmlz.F90:38-86``): primitive overlap in the radial metric,
  then ``c * 2^(l+1) sqrt(2) (2 pi)^(-3/4) * S^-1/2 * alpha^(l/2+3/4)``;
* s and p shells are Cartesian (p = x, y, z), d and higher are real spherical
  (m = -l..l) as ``Real_Sphere`` builds them
  (``gateway_util/rdctl_seward.F90:3863-3865``, ``real_spherical.F90:182``);
* AO order: shells in input order; inside a shell component-major with the
  contracted index fastest (``ao = off + m*ncontr + k``).

Generator conventions (recorded with every result): atoms uniform in a cube
of edge ``10*(N/6)^(1/3)`` bohr (the 6-atom/10-bohr number density), rejection
sampled with minimum separation 1.8 bohr; nuclear charges uniform in 1..8;
even-tempered exponents ``alpha_k = 0.08 * 3**k``, k = 0..nprim-1; general
contraction coefficients N(0,1); density ``D = C C^T``, ``C ~ N(0,1)/sqrt(r)``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List

import numpy as np

TWOP34 = 1.0 / (2.0 * math.pi) ** 0.75


def nrmlz(exps: np.ndarray, coef: np.ndarray, l: int) -> np.ndarray:
    """Normalise general-contraction coefficients (gateway_util/nrmlz.F90)."""
    exps = np.asarray(exps, dtype=np.float64)
    coef = np.array(coef, dtype=np.float64, copy=True)
    pro = np.sqrt(np.outer(exps, exps))
    s = (exps[:, None] + exps[None, :]) / 2.0
    S = (pro / s) ** (l + 1.5)
    ovl = np.einsum("pi,pq,qi->i", coef, S, coef)
    if np.any(np.abs(ovl) < 1e-12):
        raise ValueError("Nrmlz: zero column in contraction matrix")
    q = 2.0 ** (l + 1) * math.sqrt(2.0) * TWOP34
    coef = coef * q * ovl[None, :] ** -0.5 * (exps[:, None] ** (0.5 * l + 0.75))
    return coef


@dataclasses.dataclass
class Shell:
    atom: int
    l: int
    center: np.ndarray
    exps: np.ndarray
    coef: np.ndarray  # [nprim, ncontr], normalised

    @property
    def nprim(self):
        return self.exps.shape[0]

    @property
    def ncontr(self):
        return self.coef.shape[1]

    @property
    def ncomp(self):
        return 2 * self.l + 1 if self.l >= 2 else (self.l + 1) * (self.l + 2) // 2

    @property
    def nbf(self):
        return self.ncomp * self.ncontr


@dataclasses.dataclass
class Molecule:
    name: str
    coords: np.ndarray  # [natom, 3] bohr
    charges: np.ndarray  # [natom]
    shells: List[Shell]
    seed: int

    @property
    def natom(self):
        return self.coords.shape[0]

    @property
    def nbf(self):
        return sum(s.nbf for s in self.shells)

    def flat(self):
        """Plain arrays for the C ABI: xyz[nsh*3], l, nprim, ncontr, atom, exps, coefs."""
        xyz = np.concatenate([s.center for s in self.shells]).astype(np.float64)
        l = np.array([s.l for s in self.shells], dtype=np.int32)
        npr = np.array([s.nprim for s in self.shells], dtype=np.int32)
        nco = np.array([s.ncontr for s in self.shells], dtype=np.int32)
        at = np.array([s.atom for s in self.shells], dtype=np.int32)
        ex = np.concatenate([s.exps for s in self.shells]).astype(np.float64)
        cf = np.concatenate([s.coef.reshape(-1, order="F") for s in self.shells]).astype(np.float64)
        return xyz, l, npr, nco, at, ex, cf

    def at(self, coords) -> "Molecule":
        """Copy with every atom at the given coordinates (natom x 3, bohr)."""
        coords = np.array(coords, dtype=np.float64).reshape(self.natom, 3)
        shells = [dataclasses.replace(s, center=coords[s.atom].copy()) for s in self.shells]
        return Molecule(self.name, coords, self.charges, shells, self.seed)

    def moved(self, atom: int, axis: int, delta: float) -> "Molecule":
        """Copy with one atom displaced (finite-difference checks)."""
        coords = self.coords.copy()
        coords[atom, axis] += delta
        shells = [dataclasses.replace(s, center=coords[s.atom].copy()) for s in self.shells]
        return Molecule(self.name, coords, self.charges, shells, self.seed)


def _place_atoms(rng, natom, edge, dmin=1.8, max_tries=200000):
    pts = []
    tries = 0
    while len(pts) < natom:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("atom placement failed")
        p = rng.uniform(0.0, edge, 3)
        if all(np.linalg.norm(p - q) >= dmin for q in pts):
            pts.append(p)
    return np.array(pts)


def _shell(rng, atom, center, l, nprim, ncontr):
    exps = 0.08 * 3.0 ** np.arange(nprim)
    coef = rng.standard_normal((nprim, ncontr))
    return Shell(atom, l, center.copy(), exps, nrmlz(exps, coef, l))


# (ncontr, nprim) per l, "fixed" primitive sets; None = draw nprim in 1..12
BASIS_TYPES = {
    "3s2p1d": [(3, 9), (2, 4), (1, 1)],  # 3s2p1d from 9s4p1d (6-atom case)
    "2s1p": [(2, 6), (1, 3)],
    "4s3p2d": [(4, 8), (3, 5), (2, 3)],
    "4s3p2d1f": [(4, 8), (3, 5), (2, 3), (1, 1)],
    "2s1p_r": [(2, None), (1, None)],
    "4s3p2d1f_r": [(4, None), (3, None), (2, None), (1, None)],
    # large general contractions: shell pairs hold up to 450 AO pairs, above
    # the Cholesky MaxQual of 100
    "7s6p5d": [(7, 9), (6, 8), (5, 7)],
}


def make_molecule(name: str, natom: int, mix, seed: int) -> Molecule:
    """mix: list of (basis_type, count); atoms get types in a seeded shuffle."""
    rng = np.random.default_rng(seed)
    edge = 10.0 * (natom / 6.0) ** (1.0 / 3.0)
    coords = _place_atoms(rng, natom, edge)
    charges = rng.integers(1, 9, natom).astype(np.float64)
    types = []
    for t, c in mix:
        types += [t] * c
    assert len(types) == natom
    types = [types[i] for i in rng.permutation(natom)]
    shells = []
    for a in range(natom):
        for l, (nc, npr) in enumerate(BASIS_TYPES[types[a]]):
            if npr is None:
                npr = int(rng.integers(max(nc, 1), 13))
            shells.append(_shell(rng, a, coords[a], l, npr, nc))
    return Molecule(name, coords, charges, shells, seed)


CONFIGS = {
    # 6-atom cluster, 3s2p1d from 9s4p1d: 84 basis functions
    "c1": dict(natom=6, mix=[("3s2p1d", 6)], seed=1, rank=15),
    # 40 atoms, 24 x 2s1p + 16 x 4s3p2d1f, 1-12 primitives per shell: 600 bf
    "c2": dict(natom=40, mix=[("2s1p_r", 24), ("4s3p2d1f_r", 16)], seed=2, rank=60),
    # 120 atoms, 100 x 3s2p1d + 20 x 2s1p: 1500 bf
    "c3": dict(natom=120, mix=[("3s2p1d", 100), ("2s1p", 20)], seed=3, rank=200),
    # 20 atoms 4s3p2d: 460 bf
    "c4": dict(natom=20, mix=[("4s3p2d", 20)], seed=4, rank=40),
    # 250 atoms: 205 x 2s1p + 35 x 3s2p1d + 10 x 4s3p2d1f: 1815 bf
    "c5": dict(natom=250, mix=[("2s1p", 205), ("3s2p1d", 35), ("4s3p2d1f", 10)], seed=5, rank=None),
}


def config_molecule(cfg: str) -> Molecule:
    c = CONFIGS[cfg]
    return make_molecule(cfg, c["natom"], c["mix"], c["seed"])


def small_molecule(natom=3, mix=None, seed=11, name="small") -> Molecule:
    """Test-size molecule; default mixes every l up to f."""
    if mix is None:
        mix = [("4s3p2d1f_r", 1), ("2s1p", natom - 1)]
    return make_molecule(name, natom, mix, seed)


def molecule_from_arrays(name, coords, charges, shell_atom, shell_l, shell_nprim, shell_ncontr, exps,
                         coefs) -> Molecule:
    """A molecule from basis-library data: per shell its atom, l, nprim and
    ncontr; exponents concatenated; raw contraction coefficients concatenated
    per shell as [nprim, ncontr] row-major, the layout of the reference's
    basis library entries.  Coefficients are normalised with Nrmlz."""
    coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    shells = []
    pe = pc = 0
    for a, l, npr, nco in zip(shell_atom, shell_l, shell_nprim, shell_ncontr):
        a, l, npr, nco = int(a), int(l), int(npr), int(nco)
        e = np.array(exps[pe:pe + npr], dtype=np.float64)
        c = np.array(coefs[pc:pc + npr * nco], dtype=np.float64).reshape(npr, nco)
        pe += npr
        pc += npr * nco
        shells.append(Shell(a, l, coords[a].copy(), e, nrmlz(e, c, l)))
    return Molecule(name, coords, np.asarray(charges, dtype=np.float64), shells, 0)


def density_factor(nbf: int, rank: int, seed: int) -> np.ndarray:
    """C (nbf x rank, column-major contiguous as F-order) with D = C C^T."""
    rng = np.random.default_rng(1000 + seed)
    return rng.standard_normal((nbf, rank)) / math.sqrt(rank)
