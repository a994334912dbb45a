"""Python host side of libmolgpu: ctypes binding over the C ABI in
``include/molgpu.h`` plus the operator surface that mirrors the reference's
drivers (``Drv2El``/``Eval_IJKL``, ``Shell_MxSchwz``, ``Cho_Drv``,
``CHO_LK_SCF``, ``Drvg1``).

PyTorch provides device memory and streams only; every computation runs in
the hand-written kernels of ``libmolgpu.so``.  There is no CPU fallback:
without the library or a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmolgpu.so")
RYS_TABLE = os.path.join(HERE, "rys", "rys_table.bin")
# tile tables written by openmolcas_b200/autotune.py
GRAD_TILES = os.path.join(HERE, "grad_tiles.json")
ERI_TILES = os.path.join(HERE, "eri_tiles.json")

_lib = None


class MolGpuError(RuntimeError):
    pass


def lib():
    """Load libmolgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MolGpuError(f"{LIB_PATH} not built: run python -m openmolcas_b200.build")
    L = C.CDLL(LIB_PATH)
    d, i, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
    i64 = C.POINTER(C.c_int64)
    i32 = C.POINTER(C.c_int32)
    L.mg_create.argtypes = [C.c_char_p, C.c_int, C.POINTER(vp)]
    L.mg_destroy.argtypes = [vp]
    L.mg_last_error.restype = C.c_char_p
    L.mg_last_error.argtypes = [vp]
    L.mg_set_basis.argtypes = [vp, C.c_int, d, i, i, i, i, d, d]
    L.mg_nbf.argtypes = [vp]
    L.mg_natom.argtypes = [vp]
    L.mg_schwarz.argtypes = [vp, d]
    L.mg_eri_quartets_size.argtypes = [vp, i32, C.c_int64, i64]
    L.mg_eri_quartets.argtypes = [vp, i32, C.c_int64, i64, C.c_void_p, C.c_void_p]
    L.mg_cho_default.argtypes = [C.c_void_p]
    L.mg_cho_drv.argtypes = [vp, C.c_void_p, C.c_void_p]
    L.mg_cho_info.argtypes = [vp, i64, i, i]
    L.mg_cho_pivots.argtypes = [vp, i32, i32]
    L.mg_cho_rs_list.argtypes = [vp, i32, i32, i32]
    L.mg_cho_copy_vectors.argtypes = [vp, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    L.mg_cho_diag.argtypes = [vp, C.c_void_p, C.c_void_p]
    L.mg_drvg1.argtypes = [vp, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    L.mg_drvg1_x.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                             C.c_void_p]
    L.mg_cho_jk.argtypes = [vp, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.mg_rys_roots.argtypes = [vp, C.c_int, C.c_int64, d, d, d]
    L.mg_cho_jk_batch.argtypes = [vp, C.c_int, C.POINTER(C.c_void_p), i, C.POINTER(C.c_void_p),
                                  C.POINTER(C.c_void_p), C.c_int, C.c_void_p]
    L.mg_cd_incore.argtypes = [vp, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, i, C.c_void_p]
    L.mg_choscf_lk.argtypes = [vp, C.c_void_p, C.c_double, C.c_void_p, C.c_int, i, C.c_void_p]
    L.mg_eri_work.argtypes = [vp, i32, C.c_int64, d, d]
    L.mg_drvg1_flops.restype = C.c_double
    L.mg_drvg1_flops.argtypes = [vp, C.c_double]
    L.mg_grad_set_tile.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.mg_grad_profile.argtypes = [vp, C.c_int]
    L.mg_grad_class_times.argtypes = [vp, i, d, C.c_int]
    L.mg_grad_plan_info.argtypes = [vp, i, i, i, i, i, C.c_int]
    L.mg_eri_set_tile.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.mg_eri_profile.argtypes = [vp, C.c_int]
    L.mg_eri_class_times.argtypes = [vp, i, d, i, i, i, C.c_int]
    _lib = L
    return L


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class ChoCfg(C.Structure):
    """mg_cho_cfg: Cholesky thresholds (defaults of cho_inp.F90 / cholesky.F90)."""
    _fields_ = [("thrcom", C.c_double), ("span", C.c_double), ("minqual", C.c_int), ("maxqual", C.c_int),
                ("maxvec", C.c_int)]


class MolGpu:
    """One basis set resident on one GPU (the handle of the C ABI)."""

    def __init__(self, mol, device: int = 0, grad_tiles: str | None = GRAD_TILES, eri_tiles: str | None = ERI_TILES):
        """grad_tiles, eri_tiles: the tile tables to apply (the autotuner's JSON;
        None or a missing file: the planner's own choices)."""
        if not torch.cuda.is_available():
            raise MolGpuError("molgpu needs a CUDA device (no CPU fallback)")
        self.mol = mol
        self.device = device
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.mg_create(RYS_TABLE.encode(), device, C.byref(h))
        if rc != 0:
            raise MolGpuError(f"mg_create failed rc={rc}")
        self.h = h
        xyz, l, npr, nco, at, ex, cf = mol.flat()
        self._check(self.L.mg_set_basis(self.h, len(l), _p(xyz), _p(l, C.c_int), _p(npr, C.c_int), _p(nco, C.c_int),
                                        _p(at, C.c_int), _p(ex), _p(cf)), "mg_set_basis")
        self.nbf = self.L.mg_nbf(self.h)
        self.natom = self.L.mg_natom(self.h)
        self.nshell = len(l)
        if grad_tiles and os.path.exists(grad_tiles):
            with open(grad_tiles) as f:
                for key, t in json.load(f)["classes"].items():
                    nab1, ncd1 = (int(x) for x in key.split(","))
                    self.set_grad_tile(nab1, ncd1, t["tpq"], t["order"])
        if eri_tiles and os.path.exists(eri_tiles):
            with open(eri_tiles) as f:
                for key, t in json.load(f)["classes"].items():
                    nab, ncd = (int(x) for x in key.split(","))
                    self.set_eri_tile(nab, ncd, t["tpq"], t["order"])

    def _check(self, rc, what):
        if rc != 0:
            msg = self.L.mg_last_error(self.h).decode()
            raise MolGpuError(f"{what} failed rc={rc}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.mg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ ERIs
    def quartet_offsets(self, quartets: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        off = np.empty(q.shape[0] + 1, dtype=np.int64)
        self._check(self.L.mg_eri_quartets_size(self.h, _p(q, C.c_int32), q.shape[0], _p(off, C.c_int64)),
                    "mg_eri_quartets_size")
        return off

    def eri_quartets(self, quartets: np.ndarray, out: torch.Tensor | None = None):
        """Drv2El-style batch: every (i j | k l) block (i>=j, k>=l) in Eval_IJKL layout.

        Returns (device tensor of all blocks concatenated, offsets)."""
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        off = self.quartet_offsets(q)
        if out is None:
            out = torch.empty(int(off[-1]), dtype=torch.float64, device=f"cuda:{self.device}")
        self._check(self.L.mg_eri_quartets(self.h, _p(q, C.c_int32), q.shape[0], _p(off, C.c_int64),
                                           C.c_void_p(out.data_ptr()), _stream(self.device)), "mg_eri_quartets")
        return out, off

    def eval_ijkl(self, i, j, k, l):
        """One shell quartet (Eval_IJKL), flat Fortran-order AOInt(nijkl, a, b, c, d)."""
        out, _ = self.eri_quartets(np.array([[i, j, k, l]], dtype=np.int32))
        return out

    def eri_work(self, quartets: np.ndarray) -> tuple[float, float]:
        """(primitive quartets, algorithmic FP64 flops) of eri_quartets on this list."""
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        pq, fl = C.c_double(), C.c_double()
        self._check(self.L.mg_eri_work(self.h, _p(q, C.c_int32), q.shape[0], C.byref(pq), C.byref(fl)),
                    "mg_eri_work")
        return pq.value, fl.value

    def drvg1_flops(self, cutint: float = 1e-12) -> float:
        """Algorithmic FP64 flops of drvg1 at this Schwarz threshold (the
        kernel's work model over its quartet plan)."""
        f = self.L.mg_drvg1_flops(self.h, cutint)
        if f < 0:
            raise MolGpuError(f"mg_drvg1_flops: {self.L.mg_last_error(self.h).decode()}")
        return f

    def set_grad_tile(self, nab1: int, ncd1: int, tpq: int = 0, order: int = 0):
        """Tile choice of gradient class (la+lb+1, lc+ld+1): first group size
        tried (0 = the planner's) and the dimension shrunk first (0 ket
        primitives, 1 roots per wave, 2 bra primitives; 3..5 the same
        starting from 32 x 16 primitive pairs instead of 16 x 8)."""
        self._check(self.L.mg_grad_set_tile(self.h, nab1, ncd1, tpq, order), "mg_grad_set_tile")

    def grad_profile(self, enable: bool = True):
        """Later gradients run their classes one after another on the current
        stream, each timed with its own event pair."""
        self._check(self.L.mg_grad_profile(self.h, int(enable)), "mg_grad_profile")

    def grad_class_times(self) -> dict:
        """Kernel milliseconds per class (nab1, ncd1) of the last profiled gradient."""
        keys, ms = np.zeros(64, dtype=np.int32), np.zeros(64)
        n = self.L.mg_grad_class_times(self.h, _p(keys, C.c_int), _p(ms), 64)
        if n < 0:
            self._check(n, "mg_grad_class_times")
        return {(int(k) // 8, int(k) % 8): float(t) for k, t in zip(keys[:n], ms[:n])}

    def set_eri_tile(self, nab: int, ncd: int, tpq: int = 0, order: int = 0):
        """Tile choice of ERI class (la+lb, lc+ld): first group size tried (0 =
        the planner's) and the dimension shrunk first (0 ket, 1 bra primitives;
        + 2: starting from 64 x 16 primitive pairs instead of 32 x 8)."""
        self._check(self.L.mg_eri_set_tile(self.h, nab, ncd, tpq, order), "mg_eri_set_tile")

    def eri_profile(self, enable: bool = True):
        """Later ERI batches run their classes one after another on the
        current stream, each timed with its own event pair."""
        self._check(self.L.mg_eri_profile(self.h, int(enable)), "mg_eri_profile")

    def eri_class_times(self) -> dict:
        """(nab, ncd) -> (kernel ms, (tpq, pab, pcd)) of the last profiled ERI batch."""
        a = [np.zeros(64, dtype=np.int32) for _ in range(4)]
        ms = np.zeros(64)
        n = self.L.mg_eri_class_times(self.h, _p(a[0], C.c_int), _p(ms), *[_p(x, C.c_int) for x in a[1:]], 64)
        if n < 0:
            self._check(n, "mg_eri_class_times")
        return {(int(k) // 8, int(k) % 8): (float(t), (int(tq), int(pa), int(pc)))
                for k, t, tq, pa, pc in zip(a[0][:n], ms[:n], a[1][:n], a[2][:n], a[3][:n])}

    def grad_plan_info(self) -> dict:
        """Tile of every class of the current gradient plan: (tpq, pab, pcd, rw)."""
        a = [np.zeros(64, dtype=np.int32) for _ in range(5)]
        n = self.L.mg_grad_plan_info(self.h, *[_p(x, C.c_int) for x in a], 64)
        if n < 0:
            self._check(n, "mg_grad_plan_info")
        return {(int(k) // 8, int(k) % 8): (int(t), int(pa), int(pc), int(r))
                for k, t, pa, pc, r in zip(*[x[:n] for x in a])}

    def rys_roots(self, nrys: int, T) -> tuple[np.ndarray, np.ndarray]:
        """vRysRW on the device: (u^2, weights), each len(T) x nrys."""
        T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
        x = np.empty((T.size, nrys))
        w = np.empty((T.size, nrys))
        self._check(self.L.mg_rys_roots(self.h, nrys, T.size, _p(T), _p(x), _p(w)), "mg_rys_roots")
        return x, w

    def schwarz(self) -> np.ndarray:
        """Shell_MxSchwz: sqrt(max |(ab|ab)|) per shell pair (nshell x nshell)."""
        t = np.empty(self.nshell * self.nshell)
        self._check(self.L.mg_schwarz(self.h, _p(t)), "mg_schwarz")
        return t.reshape(self.nshell, self.nshell)


    # -------------------------------------------------------- Cholesky
    def cho_drv(self, thrcom: float = 1e-4, span: float = 1e-2, minqual: int = 50, maxqual: int = 100,
                maxvec: int = 0):
        """Cho_Drv (algorithm 4): decompose the ERI matrix; vectors stay on the GPU."""
        cfg = ChoCfg()
        self.L.mg_cho_default(C.byref(cfg))
        cfg.thrcom, cfg.span, cfg.minqual, cfg.maxqual, cfg.maxvec = thrcom, span, minqual, maxqual, maxvec
        self._check(self.L.mg_cho_drv(self.h, C.byref(cfg), _stream(self.device)), "mg_cho_drv")
        return self.cho_info()

    def cho_info(self):
        nrs = C.c_int64()
        nvec = C.c_int()
        npass = C.c_int()
        self._check(self.L.mg_cho_info(self.h, C.byref(nrs), C.byref(nvec), C.byref(npass)), "mg_cho_info")
        return dict(nrs=nrs.value, M=nvec.value, npass=npass.value)

    def cho_pivots(self):
        M = self.cho_info()["M"]
        piv = np.empty(M, np.int32)
        pas = np.empty(M, np.int32)
        self._check(self.L.mg_cho_pivots(self.h, _p(piv, C.c_int32), _p(pas, C.c_int32)), "mg_cho_pivots")
        return piv, pas

    def cho_rs_list(self):
        n = self.cho_info()["nrs"]
        a, b, sp = (np.empty(n, np.int32) for _ in range(3))
        self._check(self.L.mg_cho_rs_list(self.h, _p(a, C.c_int32), _p(b, C.c_int32), _p(sp, C.c_int32)),
                    "mg_cho_rs_list")
        return a, b, sp

    def cho_vectors(self, first: int = 0, count: int | None = None) -> torch.Tensor:
        """Vectors [first, first+count) as a (count, nrs) FP64 device tensor."""
        info = self.cho_info()
        if count is None:
            count = info["M"] - first
        out = torch.empty((count, info["nrs"]), dtype=torch.float64, device=f"cuda:{self.device}")
        self._check(self.L.mg_cho_copy_vectors(self.h, first, count, C.c_void_p(out.data_ptr()),
                                               _stream(self.device)), "mg_cho_copy_vectors")
        return out

    def cho_diag(self) -> torch.Tensor:
        out = torch.empty(self.cho_info()["nrs"], dtype=torch.float64, device=f"cuda:{self.device}")
        self._check(self.L.mg_cho_diag(self.h, C.c_void_p(out.data_ptr()), _stream(self.device)), "mg_cho_diag")
        return out


    # ------------------------------------------------------------- J/K
    PREC_FP64 = 0
    PREC_MIXED = 1

    @staticmethod
    def PREC_SLICED(s: int) -> int:
        """Mixed path with s 8-bit slices per operand row (2..8)."""
        return 100 + int(s)

    def cho_jk(self, Cfac: torch.Tensor, precision: int = 0, J: torch.Tensor | None = None,
               K: torch.Tensor | None = None):
        """CHO_LK_SCF for one density D = C C^T: returns (J, K), nbf x nbf device tensors."""
        dev = f"cuda:{self.device}"
        # column-major n x r == row-major r x n
        Cc = Cfac.to(device=dev, dtype=torch.float64).t().contiguous()
        n, r = self.nbf, Cfac.shape[1]
        if Cfac.shape[0] != n:
            raise MolGpuError(f"C must have {n} rows")
        if J is None:
            J = torch.empty((n, n), dtype=torch.float64, device=dev)
        if K is None:
            K = torch.empty((n, n), dtype=torch.float64, device=dev)
        self._check(self.L.mg_cho_jk(self.h, C.c_void_p(Cc.data_ptr()), r, C.c_void_p(J.data_ptr()),
                                     C.c_void_p(K.data_ptr()), precision, _stream(self.device)), "mg_cho_jk")
        return J, K

    def cho_jk_batch(self, Cfacs, precision: int = 0):
        """CHO_LK_SCF for several densities D_i = C_i C_i^T at once (1..8; every
        block of vectors is unpacked once): returns a list of (J, K)."""
        dev = f"cuda:{self.device}"
        n, k = self.nbf, len(Cfacs)
        Cc = [Cf.to(device=dev, dtype=torch.float64).t().contiguous() for Cf in Cfacs]
        for Cf in Cfacs:
            if Cf.shape[0] != n:
                raise MolGpuError(f"C must have {n} rows")
        Js = [torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(k)]
        Ks = [torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(k)]
        ptrs = lambda ts: (C.c_void_p * k)(*[t.data_ptr() for t in ts])
        rs = (C.c_int * k)(*[int(Cf.shape[1]) for Cf in Cfacs])
        self._check(self.L.mg_cho_jk_batch(self.h, k, ptrs(Cc), rs, ptrs(Js), ptrs(Ks), precision,
                                           _stream(self.device)), "mg_cho_jk_batch")
        return list(zip(Js, Ks))

    def cd_incore(self, X: torch.Tensor, thr: float = 1e-6, maxvec: int | None = None):
        """CD_InCore (cholesky_util/cd_incore.F90:14): pivoted Cholesky vectors of
        a symmetric positive semidefinite matrix X (n x n; not modified).
        Returns (Vec, irc): Vec (n x NumCho, X ~ Vec Vec^T to thr) and CD_InCore's
        return code (0; 101 a diagonal below -1e-8; 102 more than maxvec vectors)."""
        dev = f"cuda:{self.device}"
        Xc = X.to(device=dev, dtype=torch.float64).t().contiguous()  # column-major copy (overwritten)
        n = Xc.shape[0]
        maxvec = n if maxvec is None else int(maxvec)
        V = torch.zeros((max(maxvec, 1), n), dtype=torch.float64, device=dev)  # column-major n x maxvec
        nc = C.c_int(0)
        rc = self.L.mg_cd_incore(self.h, C.c_void_p(Xc.data_ptr()), n, thr, C.c_void_p(V.data_ptr()), maxvec,
                                 C.byref(nc), _stream(self.device))
        if rc not in (0, 101, 102):
            self._check(rc, "mg_cd_incore")
        return V[:nc.value].t(), rc

    def choscf_lk(self, D: torch.Tensor, factxi: float, FLT: torch.Tensor, precision: int = 0) -> int:
        """ChoSCF_Drv with the decomposed density (scf/choscf_drv.F90:99-135): D is
        cut into Cholesky vectors (CD_InCore at 1e-8 of its largest diagonal) and
        FLT += J[D] - factxi K[D] in place (FLT: nbf x nbf device tensor).
        Returns the number of density vectors."""
        dev = f"cuda:{self.device}"
        Dc = D.to(device=dev, dtype=torch.float64).contiguous()  # symmetric: layout-agnostic
        if FLT.dtype != torch.float64 or not FLT.is_contiguous() or FLT.device != torch.device(dev):
            raise MolGpuError("FLT must be a contiguous float64 tensor on the handle's device")
        nv = C.c_int(0)
        self._check(self.L.mg_choscf_lk(self.h, C.c_void_p(Dc.data_ptr()), factxi, C.c_void_p(FLT.data_ptr()),
                                        precision, C.byref(nv), _stream(self.device)), "mg_choscf_lk")
        return nv.value

    # -------------------------------------------------------- gradient
    def drvg1(self, D: torch.Tensor, cutint: float = 1e-12, out: torch.Tensor | None = None,
              exfac: float = 1.0, coulfac: float = 1.0, DS: torch.Tensor | None = None) -> torch.Tensor:
        """Drvg1: two-electron gradient dE/dR (natom x 3) of
        E = coulfac/2 tr(D J[D]) - exfac/4 (tr(D K[D]) + tr(DS K[DS])).

        The 2-PDM is PGet1's (integral_util/pget1.F90:66-110): exfac = ExFac
        (1 for Hartree-Fock, the exact-exchange fraction of a hybrid functional,
        0 for a pure one), coulfac = CoulFac, DS the spin density of an open
        shell (D_alpha - D_beta, with D = D_alpha + D_beta) or None."""
        D = D.to(device=f"cuda:{self.device}", dtype=torch.float64).contiguous()
        if D.shape != (self.nbf, self.nbf):
            raise MolGpuError(f"density must be {self.nbf}x{self.nbf}")
        ds_ptr = None
        if DS is not None:
            DS = DS.to(device=f"cuda:{self.device}", dtype=torch.float64).contiguous()
            if DS.shape != (self.nbf, self.nbf):
                raise MolGpuError(f"spin density must be {self.nbf}x{self.nbf}")
            ds_ptr = DS.data_ptr()
        if out is None:
            out = torch.empty((self.natom, 3), dtype=torch.float64, device=f"cuda:{self.device}")
        self._check(self.L.mg_drvg1_x(self.h, C.c_void_p(D.data_ptr()), C.c_void_p(ds_ptr), coulfac, exfac, cutint,
                                      C.c_void_p(out.data_ptr()), _stream(self.device)), "mg_drvg1_x")
        return out


def unique_quartets(nshell: int, tmax: np.ndarray | None = None, cutint: float = 0.0) -> np.ndarray:
    """Unique canonical quartets (i>=j, k>=l, ij>=kl) surviving Schwarz screening
    TMax(ij)*TMax(kl) >= cutint (Drv2El's pair-pair triangle, drv2el.F90:97-190)."""
    ii, jj = np.tril_indices(nshell)
    npair = ii.size
    P, Q = np.tril_indices(npair)
    if tmax is not None and cutint > 0:
        t = tmax[ii, jj]
        keep = t[P] * t[Q] >= cutint
        P, Q = P[keep], Q[keep]
    return np.stack([ii[P], jj[P], ii[Q], jj[Q]], axis=1).astype(np.int32)
