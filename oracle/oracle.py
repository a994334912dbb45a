"""ORACLE -- test infrastructure only.

ctypes wrapper around ``oracle/_build/liboracle.so`` (the CPU FP64
restatement in ``oracle.cpp``).  Imported only by ``tests/``,
``__graft_entry__.smoke()`` (as the checker) and ``bench.py``'s CPU-baseline
leg.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
# the same restatement with its FP64 operation tally compiled in
LIB_COUNT = os.path.join(HERE, "_build", "liboracle_count.so")
TABLE = os.path.join(os.path.dirname(HERE), "openmolcas_b200", "rys", "rys_table.bin")

_libs = {}

# stages of the operation tally, in or_flops order
FLOP_STAGES = ("prim", "roots", "rys2d", "rysef", "contract", "hrr", "transfer", "assg1", "pdm")


def build():
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)


def lib(counting: bool = False):
    """The oracle library; counting=True: the build that tallies its FP64
    operations (handles of one library cannot be used with the other)."""
    if counting not in _libs:
        path = LIB_COUNT if counting else LIB
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        d, i, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        L.or_load_rys.argtypes = [C.c_char_p]
        L.or_rys_rw.argtypes = [C.c_int, C.c_int, d, d, d]
        L.or_sph_matrix.argtypes = [C.c_int, d]
        L.or_basis_create.restype = vp
        L.or_basis_create.argtypes = [C.c_int, d, i, i, i, i, d, d]
        L.or_basis_free.argtypes = [vp]
        L.or_nbf.argtypes = [vp]
        L.or_eri_quartet.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, d]
        L.or_eri_quartet_abs.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, d]
        L.or_schwarz.argtypes = [vp, d]
        L.or_eri_full.argtypes = [vp, C.c_double, d]
        L.or_rs_count.restype = C.c_int64
        L.or_rs_count.argtypes = [vp]
        L.or_rs_list.argtypes = [vp, i, i, i]
        L.or_rs_compact.argtypes = [vp, C.c_double]
        L.or_eri_diag.argtypes = [vp, d]
        L.or_cholesky.argtypes = [vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, i, i, i, d, i]
        L.or_cholesky_x.argtypes = [vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i, i, i,
                                    d, i]
        L.or_cho_jk.argtypes = [vp, d, C.c_int, d, C.c_int, d, d]
        L.or_grad.argtypes = [vp, d, C.c_double, d]
        L.or_grad_x.argtypes = [vp, d, C.c_void_p, C.c_double, C.c_double, C.c_double, d]
        L.or_grad_sampled.argtypes = [vp, d, C.c_double, C.c_int, d, C.POINTER(C.c_int64)]
        L.or_grad_sampled_at.argtypes = [vp, d, C.c_double, C.c_int, C.c_int, d, C.POINTER(C.c_int64)]
        L.or_num_threads.restype = C.c_int
        L.or_flops.argtypes = [d, C.c_int]
        rc = L.or_load_rys(TABLE.encode())
        if rc != 0:
            raise RuntimeError(f"oracle: cannot load Rys table ({rc})")
        _libs[counting] = L
    return _libs[counting]


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def rys_rw(n, T):
    T = np.ascontiguousarray(T, dtype=np.float64)
    x = np.empty((T.size, n))
    w = np.empty((T.size, n))
    lib().or_rys_rw(n, T.size, _p(T), _p(x), _p(w))
    return x, w


def sph_matrix(l):
    nc = (l + 1) * (l + 2) // 2
    out = np.empty(nc * (2 * l + 1))
    lib().or_sph_matrix(l, _p(out))
    return out.reshape(2 * l + 1, nc).T


class Oracle:
    """One basis on the CPU oracle."""

    def __init__(self, mol, counting: bool = False):
        self.L = lib(counting)
        self.mol = mol
        xyz, l, npr, nco, at, ex, cf = mol.flat()
        self._keep = (xyz, l, npr, nco, at, ex, cf)
        self.h = self.L.or_basis_create(len(l), _p(xyz), _p(l, C.c_int), _p(npr, C.c_int), _p(nco, C.c_int),
                                       _p(at, C.c_int), _p(ex), _p(cf))
        self.nbf = self.L.or_nbf(self.h)
        self.nshell = len(l)

    def __del__(self):
        try:
            self.L.or_basis_free(self.h)
        except Exception:
            pass

    def flops(self, reset: bool = True) -> dict:
        """FP64 operations the counting build's loops executed since the last
        reset, per stage (FLOP_STAGES); every handle of the build shares the
        tally."""
        out = np.zeros(len(FLOP_STAGES))
        if self.L.or_flops(_p(out), int(reset)) != len(FLOP_STAGES):
            raise RuntimeError("oracle: not the counting build (Oracle(mol, counting=True))")
        return dict(zip(FLOP_STAGES, out.tolist()))

    def quartet_shape(self, i, j, k, l):
        sh = self.mol.shells
        nijkl = sh[i].ncontr * sh[j].ncontr * sh[k].ncontr * sh[l].ncontr
        return (sh[l].ncomp, sh[k].ncomp, sh[j].ncomp, sh[i].ncomp, nijkl)

    def eri_quartet(self, i, j, k, l):
        """(ij|kl) block in reference layout, returned as flat Fortran-order array."""
        shp = self.quartet_shape(i, j, k, l)
        out = np.empty(int(np.prod(shp)))
        self.L.or_eri_quartet(self.h, i, j, k, l, _p(out))
        return out

    def eri_quartet_abs(self, i, j, k, l):
        """Cancellation-free magnitude S of each integral (|coefficients|,
        |primitive [e0|f0]|, |HRR|): the scale of FP64 rounding error."""
        shp = self.quartet_shape(i, j, k, l)
        out = np.empty(int(np.prod(shp)))
        self.L.or_eri_quartet_abs(self.h, i, j, k, l, _p(out))
        return out

    def schwarz(self):
        t = np.empty(self.nshell * self.nshell)
        self.L.or_schwarz(self.h, _p(t))
        return t.reshape(self.nshell, self.nshell)

    def eri_full(self, cutint=0.0):
        n = self.nbf
        out = np.empty(n ** 4)
        self.L.or_eri_full(self.h, cutint, _p(out))
        return out.reshape(n, n, n, n)

    def rs_compact(self, thrcom):
        """Make the rs list the one a decomposition at thrcom stores its vectors
        over (the shell pairs that survive the initial screening), without
        decomposing.  A decomposition sets it as well; before either, the rs
        list holds every AO pair."""
        self.L.or_rs_compact(self.h, thrcom)

    def rs_list(self):
        """The rs list in use (AO indices a >= b within each shell pair, shell-pair id)."""
        n = self.L.or_rs_count(self.h)
        a = np.empty(n, np.int32)
        b = np.empty(n, np.int32)
        sp = np.empty(n, np.int32)
        self.L.or_rs_list(self.h, _p(a, C.c_int), _p(b, C.c_int), _p(sp, C.c_int))
        return a, b, sp

    def eri_diag(self):
        n = self.L.or_rs_count(self.h)
        d = np.empty(n)
        self.L.or_eri_diag(self.h, _p(d))
        return d

    def cholesky(self, thrcom=1e-6, span=1e-2, minqual=50, maxqual=100, maxvec=None, mxshpr=1, ialqua=2):
        """Pivoted Cholesky decomposition.  mxshpr/ialqua: shell pairs per pass
        and qualification algorithm; (1, 2) is the reference's default for
        algorithm 4 and what the device decomposition implements."""
        nrs = self.nbf * (self.nbf + 1) // 2  # every AO pair: the bound of the decomposition's rs list
        if maxvec is None:
            maxvec = min(nrs, 20 * self.nbf)
        L = np.zeros(nrs * maxvec)
        piv = np.zeros(maxvec, np.int32)
        pas = np.zeros(maxvec, np.int32)
        M = C.c_int(0)
        npass = C.c_int(0)
        rc = self.L.or_cholesky_x(self.h, thrcom, span, minqual, maxqual, mxshpr, ialqua, maxvec, C.byref(M),
                                 _p(piv, C.c_int), _p(pas, C.c_int), _p(L), C.byref(npass))
        if rc != 0:
            raise RuntimeError(f"oracle cholesky failed rc={rc}")
        m = M.value
        nrs = self.L.or_rs_count(self.h)  # the decomposition's rs list (screened shell pairs have no rows)
        return dict(L=L[: nrs * m].reshape(m, nrs).T.copy(), piv=piv[:m].copy(), pass_of=pas[:m].copy(),
                    M=m, npass=npass.value)

    def cho_jk(self, L, Cm):
        nrs, M = L.shape
        Lf = np.asfortranarray(L)
        Cf = np.asfortranarray(Cm, dtype=np.float64)
        n = self.nbf
        J = np.empty(n * n)
        K = np.empty(n * n)
        self.L.or_cho_jk(self.h, _p(Lf), M, _p(Cf), Cf.shape[1], _p(J), _p(K))
        return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")

    def grad(self, D, cutint=0.0, exfac=1.0, coulfac=1.0, DS=None):
        Dc = np.ascontiguousarray(D, dtype=np.float64)
        Ds = None if DS is None else np.ascontiguousarray(DS, dtype=np.float64)
        g = np.empty(3 * self.mol.natom)
        self.L.or_grad_x(self.h, _p(Dc), None if Ds is None else Ds.ctypes.data, coulfac, exfac, cutint, _p(g))
        return g.reshape(-1, 3)


# FP64 parity bar of one integral: 1e-11 absolute plus a rounding term scaled
# by the integral's cancellation-free magnitude S (random-sign general
# contractions over exponents spanning 4 decades cancel by up to ~1e7).
ERI_ABS_TOL = 1e-11
ERI_REL_S = 1e-13


def eri_tolerance(S):
    return ERI_ABS_TOL + ERI_REL_S * S


def grad_sampled(orc, D, cutint, stride, offset=0):
    """Oracle gradient over every stride-th unique quartet starting at
    `offset`; returns (grad, nquartets)."""
    Dc = np.ascontiguousarray(D, dtype=np.float64)
    g = np.empty(3 * orc.mol.natom)
    nq = C.c_int64(0)
    orc.L.or_grad_sampled_at(orc.h, _p(Dc), cutint, stride, offset % stride, _p(g), C.byref(nq))
    return g.reshape(-1, 3), nq.value


def cho_jk_blas(rs_a, rs_b, n, L, Cm, batch=16):
    """CHO_LK_SCF's J and K without screening, driven through numpy's BLAS the
    way the reference drives its linked BLAS: V = L^T d and J = L V as DGEMV
    (fock_util/cho_lk_scf.F90:442-449), X_J = L_J C as DGEMM and K += X X^T as
    DGEMM (:507-830).  L: vectors (nrs x M) in the rs order (rs_a, rs_b);
    Cm: density factor (n x r).  Returns J, K (n x n).  Used as the timed CPU
    baseline of the exchange build (cost does not depend on the values)."""
    rs_a = np.asarray(rs_a, dtype=np.int64)
    rs_b = np.asarray(rs_b, dtype=np.int64)
    D = Cm @ Cm.T
    w = np.where(rs_a == rs_b, 1.0, 2.0) * D[rs_a, rs_b]
    V = L.T @ w
    Jrs = L @ V
    K = np.zeros((n, n))
    M = L.shape[1]
    for J0 in range(0, M, batch):
        Lb = L[:, J0:J0 + batch].T
        Lsq = np.zeros((Lb.shape[0], n, n))
        Lsq[:, rs_a, rs_b] = Lb
        Lsq[:, rs_b, rs_a] = Lb
        X = np.matmul(Lsq, Cm)
        Xa = X.transpose(1, 0, 2).reshape(n, -1)
        K += Xa @ Xa.T
    J = np.zeros((n, n))
    J[rs_a, rs_b] = Jrs
    J[rs_b, rs_a] = Jrs
    return J, K


def cd_incore(X, thr=1e-6, maxvec=None):
    """CD_InCore restated (cholesky_util/cd_incore.F90:14-44 and
    cd_incore_1.F90:14-100): left-looking pivoted Cholesky of a symmetric
    positive semidefinite matrix with the reference's pivot rule (the first
    diagonal, in index order, above the running maximum + Acc,
    Acc = min(1e-12, Thr/100)), ThrNeg = -1e-13 (zero the row and column),
    ThrFail = -1e-8 (irc 101), MxVec (irc 102).  Returns (Vec, irc)."""
    X = np.array(X, dtype=np.float64, copy=True)
    n = X.shape[0]
    if thr < 0.0:
        thr = 1e-6
    maxvec = n if maxvec is None else maxvec
    vec = np.zeros((n, maxvec))
    acc = min(1e-12, thr * 1e-2)
    numcho = 0
    for _ in range(n):
        xmax, imax = 0.0, -1
        for i in range(n):
            if X[i, i] < -1e-13:
                if X[i, i] < -1e-8:
                    return vec[:, :numcho], 101
                X[:, i] = 0.0
                X[i, :] = 0.0
            if X[i, i] > xmax + acc:
                xmax, imax = X[i, i], i
        if xmax <= thr:
            return vec[:, :numcho], 0
        if numcho == maxvec:
            return vec[:, :numcho], 102
        xfac = 1.0 / np.sqrt(abs(xmax))
        for j in range(numcho):
            X[:, imax] -= vec[imax, j] * vec[:, j]
        X[imax, imax] = xmax
        d = np.diagonal(X).copy()
        vec[:, numcho] = np.where(d == 0.0, 0.0, xfac * X[:, imax])
        numcho += 1
        X[np.arange(n), np.arange(n)] -= vec[:, numcho - 1] ** 2
        X[imax, imax] = 0.0
    return vec[:, :numcho], 0


def num_threads():
    return lib().or_num_threads()


def energy_from_full(eri, D):
    """E = 1/2 tr(DJ) - 1/4 tr(DK) from a full ERI tensor."""
    J = np.einsum("abcd,cd->ab", eri, D)
    K = np.einsum("acbd,cd->ab", eri, D)
    return 0.5 * np.sum(D * J) - 0.25 * np.sum(D * K), J, K
