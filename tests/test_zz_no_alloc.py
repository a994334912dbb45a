"""The allocation-free ERI entry point (mg_eri_quartets_noalloc).

It exists for callers that cannot let the library allocate device memory
during a call (all device memory reserved up front by the caller's own pool
or a framework's caching allocator, or no device-wide synchronisation from
cudaFree allowed).  It must give the same integrals as mg_eri_quartets, call
after call, although every call reuses the same fixed device array.  This
file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, lib, unique_quartets

pytestmark = pytest.mark.gpu


def _noalloc():
    f = lib().mg_eri_quartets_noalloc
    f.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _call(g, f, q, off, out):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return f(g.h, q.ctypes.data_as(C.POINTER(C.c_int32)), q.shape[0], off.ctypes.data_as(C.POINTER(C.c_int64)),
             C.c_void_p(out.data_ptr()), stream)


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    mol = B.small_molecule(3, seed=5)
    g = MolGpu(mol)
    q = np.ascontiguousarray(unique_quartets(len(mol.shells)), dtype=np.int32)
    ref, off = g.eri_quartets(q)
    torch.cuda.synchronize()
    f = _noalloc()
    for _ in range(2):
        out = torch.full_like(ref, float("nan"))
        rc = _call(g, f, q, off, out)
        torch.cuda.synchronize()
        assert rc == 0, lib().mg_last_error(g.h)
        assert not torch.isnan(out).any()
        assert float((out - ref).abs().max()) <= O.ERI_ABS_TOL


def test_noalloc_rejects_more_items_than_its_capacity():
    mol = B.small_molecule(3, seed=5)
    g = MolGpu(mol)
    q1 = unique_quartets(len(mol.shells))
    q = np.ascontiguousarray(np.tile(q1, (70000 // len(q1) + 1, 1)), dtype=np.int32)
    off = g.quartet_offsets(q)
    out = torch.empty(int(off[-1]), dtype=torch.float64, device="cuda")
    rc = _call(g, _noalloc(), q, off, out)
    assert rc != 0
    assert b"capacity" in lib().mg_last_error(g.h)
