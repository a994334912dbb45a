"""Cho_Qualify_2 as the device decomposition runs it between passes
(openmolcas_b200/csrc/cho_qualify.h, host C++), compiled here with g++ and
checked against a restatement of cholesky_util/cho_qualify_2.F90 on random
shell pairs: more candidates than MaxQual (the replacement branch), MaxQual 1,
ties, entries outside the reduced set and below DiaMin."""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "openmolcas_b200", "csrc")

DRIVER = r"""
#include "cho_qualify.h"
extern "C" int qualify(const double* d, const unsigned char* r, int cnt, double diamin, int maxqual, int* out) {
  std::vector<int> q = mg::cho_qualify_2(d, r, cnt, diamin, maxqual);
  for (size_t i = 0; i < q.size(); ++i) out[i] = q[i];
  return (int)q.size();
}
"""


def qualify_ref(d, r, diamin, maxq):
    """cho_qualify_2.F90 for one symmetry, the shell pair's rows in order."""
    if maxq == 1:  # the largest >= DIAMIN; '>=' keeps the last of equal ones
        xmax, imax = diamin, -1
        for i in range(len(d)):
            if r[i] and d[i] >= xmax:
                xmax, imax = d[i], i
        return [imax] if imax >= 0 else []
    q = []
    for i in range(len(d)):
        if not (r[i] and d[i] >= diamin):
            continue
        if len(q) < maxq:
            q.append(i)
        else:  # replace the first smallest if the new one is larger
            kmin = min(range(len(q)), key=lambda k: (d[q[k]], k))
            if d[i] > d[q[kmin]]:
                q[kmin] = i
    return q


def test_device_qualification_matches_cho_qualify_2(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    lib = tmp_path / "libqual.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", HEADER_DIR, str(src), "-o", str(lib)],
                   check=True)
    L = C.CDLL(str(lib))
    L.qualify.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_ubyte), C.c_int, C.c_double, C.c_int,
                          C.POINTER(C.c_int)]
    rng = np.random.default_rng(7)
    nrep = 0
    for case in range(400):
        cnt = int(rng.integers(1, 480))
        d = rng.choice([0.0, 1e-3, 2e-3, 5e-2, 0.3, 0.3, 1.0], cnt) if case % 3 == 0 else rng.random(cnt)
        d = np.ascontiguousarray(d, dtype=np.float64)
        r = np.ascontiguousarray((rng.random(cnt) < 0.85).astype(np.uint8))
        diamin = float(rng.choice([1e-3, 0.05, 0.2]))
        maxq = int(rng.choice([1, 2, 7, 50, 100]))
        out = np.empty(max(maxq, 1), np.int32)
        n = L.qualify(d.ctypes.data_as(C.POINTER(C.c_double)), r.ctypes.data_as(C.POINTER(C.c_ubyte)), cnt,
                      diamin, maxq, out.ctypes.data_as(C.POINTER(C.c_int)))
        ref = qualify_ref(d, r, diamin, maxq)
        assert out[:n].tolist() == ref, (case, cnt, maxq)
        ncand = int(np.sum((r > 0) & (d >= diamin)))
        nrep += maxq > 1 and ncand > maxq
    assert nrep > 50  # the replacement branch ran
