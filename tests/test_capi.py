"""CPU checks of the C ABI: the library builds/loads and exports every
function include/molgpu.h declares (no compute calls: no GPU here)."""
import ctypes
import os
import re

from openmolcas_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "molgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    lib = build.build()
    L = ctypes.CDLL(lib)
    syms = declared_symbols()
    assert len(syms) >= 8
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_create_rejects_bad_arguments_without_gpu():
    L = ctypes.CDLL(build.build())
    L.mg_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p]
    assert L.mg_create(None, 0, None) != 0
