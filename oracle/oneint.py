"""ORACLE -- test infrastructure only.

One-electron integrals (overlap, kinetic energy, nuclear attraction) in the
basis conventions of the two-electron oracle, so that a whole RHF energy can
be checked against values the reference prints.  The reference computes these
in Seward (``integral_util/oneel.F90``: the 'Kinetic ' and 'Attract ' labels,
the point-charge attraction of every nucleus); this file restates the same
matrices with published recurrences of its own choosing:

* overlap and kinetic energy: Obara--Saika 1D recurrences
  (S. Obara, A. Saika, J. Chem. Phys. 84 (1986) 3963), T by the 1D identity
  T_ij = -2 b^2 S_i,j+2 + b (2j+1) S_ij - j(j-1)/2 S_i,j-2;
* nuclear attraction: McMurchie--Davidson Hermite expansion
  (L. E. McMurchie, E. R. Davidson, J. Comput. Phys. 26 (1978) 218) with the
  Boys function from the regularised lower incomplete gamma function.

Conventions shared with ``oracle.cpp`` (and therefore with the reference):
unnormalised Cartesian primitives x^lx y^ly z^lz exp(-a r^2), Cartesian order
lx = l..0 then ly = l-lx..0; Nrmlz-normalised general contraction coefficients
(``Shell.coef``); s and p Cartesian (p = x, y, z), d and higher transformed by
the oracle's Real_Sphere matrix (m = -l..l); AO order component-major with the
contracted index fastest.  Imported only by tests.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import gammainc

from . import oracle as O


def _carts(l):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def boys(nmax, T):
    """F_n(T), n = 0..nmax: gamma(n+1/2) P(n+1/2, T) / (2 T^(n+1/2))."""
    if T < 1e-12:
        return np.array([1.0 / (2 * n + 1) - T / (2 * n + 3) for n in range(nmax + 1)])
    n = np.arange(nmax + 1) + 0.5
    g = np.array([math.gamma(v) for v in n])
    return g * gammainc(n, T) / (2.0 * T ** n)


def _os_1d(la, lb, PA, PB, p, s00):
    """S[i][j], i <= la, j <= lb, one Cartesian direction (Obara-Saika)."""
    S = np.zeros((la + 1, lb + 1))
    S[0, 0] = s00
    h = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                v = PA * S[i - 1, j]
                if i > 1:
                    v += (i - 1) * h * S[i - 2, j]
                if j > 0:
                    v += j * h * S[i - 1, j - 1]
            else:
                v = PB * S[i, j - 1]
                if j > 1:
                    v += (j - 1) * h * S[i, j - 2]
            S[i, j] = v
    return S


def _hermite_1d(la, lb, PA, PB, p, e00):
    """E[i][j][t] of the McMurchie-Davidson expansion in one direction."""
    E = np.zeros((la + 1, lb + 1, la + lb + 2))
    E[0, 0, 0] = e00
    h = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                src, X = E[i - 1, j], PA
            else:
                src, X = E[i, j - 1], PB
            for t in range(i + j + 1):
                v = X * src[t]
                if t > 0:
                    v += h * src[t - 1]
                if t + 1 < src.shape[0]:
                    v += (t + 1) * src[t + 1]
                E[i, j, t] = v
    return E


def _hermite_r(L, p, PC):
    """R[t][u][v] = R^0_tuv(p, PC) for t + u + v <= L."""
    T = p * float(PC @ PC)
    F = boys(L, T)
    Rn = np.zeros((L + 1, L + 1, L + 1, L + 1))  # [n][t][u][v]
    for n in range(L + 1):
        Rn[n, 0, 0, 0] = (-2.0 * p) ** n * F[n]
    X, Y, Z = PC
    for tot in range(1, L + 1):
        for n in range(L - tot + 1):
            for t in range(tot + 1):
                for u in range(tot - t + 1):
                    v = tot - t - u
                    if t > 0:
                        r = X * Rn[n + 1, t - 1, u, v] + ((t - 1) * Rn[n + 1, t - 2, u, v] if t > 1 else 0.0)
                    elif u > 0:
                        r = Y * Rn[n + 1, t, u - 1, v] + ((u - 1) * Rn[n + 1, t, u - 2, v] if u > 1 else 0.0)
                    else:
                        r = Z * Rn[n + 1, t, u, v - 1] + ((v - 1) * Rn[n + 1, t, u, v - 2] if v > 1 else 0.0)
                    Rn[n, t, u, v] = r
    return Rn[0]


def _prim_block(sa, sb, ka, kb, nuclei):
    """Cartesian primitive blocks S, T, V for primitives ka of sa and kb of sb."""
    a, b = sa.exps[ka], sb.exps[kb]
    A, B = sa.center, sb.center
    p = a + b
    P = (a * A + b * B) / p
    mu = a * b / p
    AB = A - B
    la, lb = sa.l, sb.l
    Sx = [_os_1d(la, lb + 2, P[d] - A[d], P[d] - B[d], p, math.sqrt(math.pi / p) * math.exp(-mu * AB[d] ** 2))
          for d in range(3)]
    Tx = []
    for d in range(3):
        S = Sx[d]
        T = np.zeros((la + 1, lb + 1))
        for i in range(la + 1):
            for j in range(lb + 1):
                v = -2.0 * b * b * S[i, j + 2] + b * (2 * j + 1) * S[i, j]
                if j > 1:
                    v -= 0.5 * j * (j - 1) * S[i, j - 2]
                T[i, j] = v
        Tx.append(T)
    Ex = [_hermite_1d(la, lb, P[d] - A[d], P[d] - B[d], p, math.exp(-mu * AB[d] ** 2)) for d in range(3)]
    ca, cb = _carts(la), _carts(lb)
    Sm = np.zeros((len(ca), len(cb)))
    Tm = np.zeros_like(Sm)
    Vm = np.zeros_like(Sm)
    Rs = [(Z, _hermite_r(la + lb, p, P - C)) for Z, C in nuclei]
    for u, (ax, ay, az) in enumerate(ca):
        for v, (bx, by, bz) in enumerate(cb):
            sx, sy, sz = Sx[0][ax, bx], Sx[1][ay, by], Sx[2][az, bz]
            Sm[u, v] = sx * sy * sz
            Tm[u, v] = Tx[0][ax, bx] * sy * sz + sx * Tx[1][ay, by] * sz + sx * sy * Tx[2][az, bz]
            ex, ey, ez = Ex[0][ax, bx], Ex[1][ay, by], Ex[2][az, bz]
            acc = 0.0
            for Z, R in Rs:
                s = 0.0
                for t in range(ax + bx + 1):
                    for w in range(ay + by + 1):
                        s += ex[t] * ey[w] * float(ez[: az + bz + 1] @ R[t, w, : az + bz + 1])
                acc -= Z * s
            Vm[u, v] = 2.0 * math.pi / p * acc
    return Sm, Tm, Vm


def one_electron(mol):
    """(S, T, V) nbf x nbf in the molecule's AO basis; V sums every nucleus."""
    nuclei = [(float(mol.charges[i]), np.asarray(mol.coords[i], dtype=np.float64)) for i in range(mol.natom)]
    offs = np.cumsum([0] + [s.nbf for s in mol.shells])
    n = int(offs[-1])
    out = [np.zeros((n, n)) for _ in range(3)]
    sph = {}

    def tr(l):
        if l < 2:
            return np.eye((l + 1) * (l + 2) // 2)
        if l not in sph:
            sph[l] = O.sph_matrix(l)  # ncart x (2l+1)
        return sph[l]

    for i, sa in enumerate(mol.shells):
        for j, sb in enumerate(mol.shells):
            if j > i:
                continue
            nca, ncb = len(_carts(sa.l)), len(_carts(sb.l))
            acc = [np.zeros((nca, sa.ncontr, ncb, sb.ncontr)) for _ in range(3)]
            for ka in range(sa.nprim):
                for kb in range(sb.nprim):
                    blocks = _prim_block(sa, sb, ka, kb, nuclei)
                    cc = np.outer(sa.coef[ka], sb.coef[kb])  # [ncontr_a, ncontr_b]
                    for m in range(3):
                        acc[m] += blocks[m][:, None, :, None] * cc[None, :, None, :]
            Ua, Ub = tr(sa.l), tr(sb.l)
            for m in range(3):
                blk = np.einsum("ucvd,um,vn->mcnd", acc[m], Ua, Ub)  # component-major, contracted fastest
                blk = blk.reshape(sa.nbf, sb.nbf)
                out[m][offs[i]:offs[i + 1], offs[j]:offs[j + 1]] = blk
                out[m][offs[j]:offs[j + 1], offs[i]:offs[i + 1]] = blk.T
    return tuple(out)


def nuclear_repulsion(mol):
    e = 0.0
    for i in range(mol.natom):
        for j in range(i):
            e += mol.charges[i] * mol.charges[j] / float(np.linalg.norm(mol.coords[i] - mol.coords[j]))
    return e


def _prim_tables(sa, sb, ka, kb, nuclei, extra):
    """1D tables of one primitive pair with angular momenta raised by
    ``extra`` (1 for first derivatives): S and T per direction, the Hermite
    expansion per direction and R_tuv per nucleus."""
    a, b = sa.exps[ka], sb.exps[kb]
    A, B = sa.center, sb.center
    p = a + b
    P = (a * A + b * B) / p
    mu = a * b / p
    AB = A - B
    la, lb = sa.l + extra, sb.l + extra
    Sx = [_os_1d(la, lb + 2, P[d] - A[d], P[d] - B[d], p, math.sqrt(math.pi / p) * math.exp(-mu * AB[d] ** 2))
          for d in range(3)]
    Tx = []
    for d in range(3):
        S = Sx[d]
        T = np.zeros((la + 1, lb + 1))
        for i in range(la + 1):
            for j in range(lb + 1):
                v = -2.0 * b * b * S[i, j + 2] + b * (2 * j + 1) * S[i, j]
                if j > 1:
                    v -= 0.5 * j * (j - 1) * S[i, j - 2]
                T[i, j] = v
        Tx.append(T)
    Ex = [_hermite_1d(la, lb, P[d] - A[d], P[d] - B[d], p, math.exp(-mu * AB[d] ** 2)) for d in range(3)]
    Rs = [_hermite_r(la + lb, p, P - C) for _, C in nuclei]
    return a, b, p, Sx, Tx, Ex, Rs


def _ints(tab, u, v, nuclei):
    """S, T and V_C (per nucleus, without -Z) of Cartesian exponent triples u, v."""
    a, b, p, Sx, Tx, Ex, Rs = tab
    if min(u) < 0 or min(v) < 0:
        return 0.0, 0.0, np.zeros(len(nuclei))
    sx, sy, sz = Sx[0][u[0], v[0]], Sx[1][u[1], v[1]], Sx[2][u[2], v[2]]
    s = sx * sy * sz
    t = Tx[0][u[0], v[0]] * sy * sz + sx * Tx[1][u[1], v[1]] * sz + sx * sy * Tx[2][u[2], v[2]]
    ex, ey, ez = Ex[0][u[0], v[0]], Ex[1][u[1], v[1]], Ex[2][u[2], v[2]]
    vc = np.empty(len(nuclei))
    for c, R in enumerate(Rs):
        acc = 0.0
        for tt in range(u[0] + v[0] + 1):
            for w in range(u[1] + v[1] + 1):
                acc += ex[tt] * ey[w] * float(ez[: u[2] + v[2] + 1] @ R[tt, w, : u[2] + v[2] + 1])
        vc[c] = 2.0 * math.pi / p * acc
    return s, t, vc


def one_electron_gradient(mol, D, W):
    """sum_mn D_mn dh_mn/dR - W_mn dS_mn/dR (natom x 3), h = T + V.

    The derivative of a primitive with respect to its centre is
    2 alpha |u + e_d> - u_d |u - e_d>; the operator (Hellmann-Feynman) part of
    the attraction of nucleus C follows from translational invariance:
    d<a|V_C|b>/dC = -(d/dA + d/dB)<a|V_C|b>.  D, W: full symmetric AO
    matrices (density and energy-weighted density)."""
    nuclei = [(float(mol.charges[i]), np.asarray(mol.coords[i], dtype=np.float64)) for i in range(mol.natom)]
    offs = np.cumsum([0] + [s.nbf for s in mol.shells])
    G = np.zeros((mol.natom, 3))
    sph = {}

    def tr(l):
        if l < 2:
            return np.eye((l + 1) * (l + 2) // 2)
        if l not in sph:
            sph[l] = O.sph_matrix(l)
        return sph[l]

    for i, sa in enumerate(mol.shells):
        for j, sb in enumerate(mol.shells):
            ca, cb = _carts(sa.l), _carts(sb.l)
            # accumulators [type][d]: dS/dA, dS/dB, dT/dA, dT/dB, (unused 4, 5), dV_C/dA per C, dV_C/dB per C
            nC = len(nuclei)
            acc = np.zeros((6 + 2 * nC, 3, len(ca), sa.ncontr, len(cb), sb.ncontr))
            for ka in range(sa.nprim):
                for kb in range(sb.nprim):
                    tab = _prim_tables(sa, sb, ka, kb, nuclei, 1)
                    a, b = tab[0], tab[1]
                    cc = np.outer(sa.coef[ka], sb.coef[kb])
                    for u, ue in enumerate(ca):
                        for v, ve in enumerate(cb):
                            for d in range(3):
                                up = list(ue); up[d] += 1
                                um = list(ue); um[d] -= 1
                                vp = list(ve); vp[d] += 1
                                vm = list(ve); vm[d] -= 1
                                sp, tp, vpc = _ints(tab, up, ve, nuclei)
                                sm, tm, vmc = _ints(tab, um, ve, nuclei)
                                dA = (2 * a * sp - ue[d] * sm, 2 * a * tp - ue[d] * tm, 2 * a * vpc - ue[d] * vmc)
                                sp, tp, vpc = _ints(tab, ue, vp, nuclei)
                                sm, tm, vmc = _ints(tab, ue, vm, nuclei)
                                dB = (2 * b * sp - ve[d] * sm, 2 * b * tp - ve[d] * tm, 2 * b * vpc - ve[d] * vmc)
                                acc[0, d, u, :, v, :] += dA[0] * cc
                                acc[1, d, u, :, v, :] += dB[0] * cc
                                acc[2, d, u, :, v, :] += dA[1] * cc
                                acc[3, d, u, :, v, :] += dB[1] * cc
                                for c in range(nC):
                                    acc[6 + c, d, u, :, v, :] += dA[2][c] * cc
                                    acc[6 + nC + c, d, u, :, v, :] += dB[2][c] * cc
            Ua, Ub = tr(sa.l), tr(sb.l)
            blkD = D[offs[i]:offs[i + 1], offs[j]:offs[j + 1]]
            blkW = W[offs[i]:offs[i + 1], offs[j]:offs[j + 1]]

            def contract(m, d):
                return np.einsum("ucvd,um,vn->mcnd", acc[m, d], Ua, Ub).reshape(sa.nbf, sb.nbf)

            for d in range(3):
                dSA, dSB = contract(0, d), contract(1, d)
                dTA, dTB = contract(2, d), contract(3, d)
                G[sa.atom, d] += np.sum(blkD * dTA) - np.sum(blkW * dSA)
                G[sb.atom, d] += np.sum(blkD * dTB) - np.sum(blkW * dSB)
                for c, (Z, _) in enumerate(nuclei):
                    dVA, dVB = contract(6 + c, d), contract(6 + nC + c, d)
                    eA, eB = -Z * np.sum(blkD * dVA), -Z * np.sum(blkD * dVB)
                    G[sa.atom, d] += eA
                    G[sb.atom, d] += eB
                    G[c, d] -= eA + eB
    return G


def nuclear_repulsion_gradient(mol):
    G = np.zeros((mol.natom, 3))
    for i in range(mol.natom):
        for j in range(mol.natom):
            if i != j:
                r = mol.coords[i] - mol.coords[j]
                G[i] -= mol.charges[i] * mol.charges[j] * r / float(np.linalg.norm(r)) ** 3
    return G
