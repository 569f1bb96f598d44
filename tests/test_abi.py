"""CPU tests of the drop-in boundary: the C-ABI library loads and exports every
symbol include/*.h declares (no compute calls without a GPU)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "qumasun-workshop-template_b200", "libqumasun_b200.so")


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        names.update(re.findall(r"QSB_API\s+[\w\s\*]*?\b(qsb_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "qsb_ham_apply" in syms and "qsb_laplacian8th" in syms
    assert len(syms) >= 13


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build with python qumasun-workshop-template_b200/build_lib.py"
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_exports_nothing_undeclared():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and l.split()[-1].startswith("qsb_")}
    assert exported == set(declared_symbols())


def test_version_and_error_strings():
    lib = ctypes.CDLL(LIB)
    lib.qsb_version.restype = ctypes.c_char_p
    lib.qsb_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.qsb_version()
    # an argument error is reported without touching the GPU
    st = lib.qsb_laplacian8th(0, 0, 4, 4, 1, None, None, ctypes.c_double(1.0), ctypes.c_double(1.0),
                              ctypes.c_double(1.0), ctypes.c_double(1.0), None)
    assert st == 1 and b"grid" in lib.qsb_last_error()
