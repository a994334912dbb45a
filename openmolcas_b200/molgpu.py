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
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmolgpu.so")
RYS_TABLE = os.path.join(HERE, "rys", "rys_table.bin")

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
    _lib = L
    return L


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class MolGpu:
    """One basis set resident on one GPU (the handle of the C ABI)."""

    def __init__(self, mol, device: int = 0):
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

    def schwarz(self) -> np.ndarray:
        """Shell_MxSchwz: sqrt(max |(ab|ab)|) per shell pair (nshell x nshell)."""
        t = np.empty(self.nshell * self.nshell)
        self._check(self.L.mg_schwarz(self.h, _p(t)), "mg_schwarz")
        return t.reshape(self.nshell, self.nshell)


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
