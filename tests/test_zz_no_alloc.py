"""The allocation-free ERI entry point (mg_eri_quartets_noalloc).

It exists for callers that cannot let the library allocate device memory
during a call (all device memory reserved up front by the caller's own pool
or a framework's caching allocator, or no device-wide synchronisation from
cudaFree allowed).  It must give the same integrals as mg_eri_quartets, call
after call, although every call reuses the same fixed device array, and it
must not allocate even when it is the first ERI call of a process.  This
file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from oracle import oracle as O
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, lib, unique_quartets

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _noalloc():
    f = lib().mg_eri_quartets_noalloc
    f.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _call(g, f, q, off, out):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return f(g.h, q.ctypes.data_as(C.POINTER(C.c_int32)), q.shape[0], off.ctypes.data_as(C.POINTER(C.c_int64)),
             C.c_void_p(out.data_ptr()), stream)


def _allocs():
    f = lib().mg_device_allocations
    f.restype = C.c_longlong
    return int(f())


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


_FRESH = r"""
import json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from tests.test_zz_no_alloc import _noalloc, _call, _allocs
from openmolcas_b200 import basis as B
from openmolcas_b200.molgpu import MolGpu, unique_quartets
mol = B.small_molecule(3, seed=5)
g = MolGpu(mol)
q = np.ascontiguousarray(unique_quartets(len(mol.shells)), dtype=np.int32)
off = g.quartet_offsets(q)
outs = [torch.full((int(off[-1]),), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
torch.cuda.synchronize()
f = _noalloc()
rec = []
for out in outs:
    a0, free0 = _allocs(), torch.cuda.mem_get_info()[0]
    rc = _call(g, f, q, off, out)
    torch.cuda.synchronize()
    rec.append(dict(rc=rc, allocs=_allocs() - a0, freed=free0 - torch.cuda.mem_get_info()[0]))
ref, _ = g.eri_quartets(q)
torch.cuda.synchronize()
diff = [float((o - ref).abs().max()) for o in outs]
print(json.dumps(dict(calls=rec, diff=diff)))
"""


def test_noalloc_first_call_of_a_process_allocates_nothing():
    """In a fresh process whose first ERI call is the allocation-free one: the
    library's allocation counter does not move over either of two calls, the
    device's free memory does not change (modules are loaded eagerly at
    context creation, so only an allocation could change it), and both calls
    give the integrals of the allocating entry point."""
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    for c in res["calls"]:
        assert c["rc"] == 0
        assert c["allocs"] == 0
        assert c["freed"] == 0
    assert max(res["diff"]) <= O.ERI_ABS_TOL
