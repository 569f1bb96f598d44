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


DROPIN_PROGRAM = r"""
#include <cstdio>
#include <cstddef>
struct GridRange { int begin_x, begin_y, begin_z, end_x, end_y, end_z;
  int SizeX() const { return end_x - begin_x; } int SizeY() const { return end_y - begin_y; }
  int SizeZ() const { return end_z - begin_z; } };
struct SoAComplex { double* re; double* im; };
struct OneComplex { double r, i; };
#include "qumasun_dropin.hpp"
struct W { void Record(int) {} };
int main() {
  GridRange g{0, 0, 0, 8, 8, 8};
  qsb_dropin::Hamiltonian H(g, 0.5, 0.5, 0.5);          // host-side context, no GPU work
  GridRange bad{0, 0, 0, 0, 8, 8};
  try { qsb_dropin::Laplacian8th<double>(bad, nullptr, nullptr, -0.5, 0.5, 0.5, 0.5); }
  catch (const std::exception& e) { std::printf("caught: %s\n", e.what()); return 0; }
  return 1;
}
"""


def test_dropin_header_compiles_and_reports_errors(tmp_path):
    """The reference-signature adapter header compiles against reference-style
    types, links to the library and turns an error status into an exception."""
    src = tmp_path / "dropin.cpp"
    src.write_text(DROPIN_PROGRAM)
    exe = tmp_path / "dropin"
    libdir = os.path.dirname(LIB)
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lqumasun_b200", f"-Wl,-rpath,{libdir}"], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "grid dimensions" in out.stdout


def test_host_side_argument_errors_of_the_newer_entry_points():
    """Argument and state errors are reported before any device work, so they
    are checked without a GPU: the kinetic switch, the host-buffer apply, the
    Ewald sum and the relaxation driver."""
    lib = ctypes.CDLL(LIB)
    lib.qsb_last_error.restype = ctypes.c_char_p
    d = ctypes.c_double
    h = ctypes.c_void_p()
    assert lib.qsb_ham_create(ctypes.byref(h), 8, 8, 8, d(0.5), d(0.5), d(0.5)) == 0
    try:
        assert lib.qsb_ham_set_kinetic(h, 2) == 1 and b"FD8" in lib.qsb_last_error()
        assert lib.qsb_ham_set_kinetic(h, 1) == 0 and lib.qsb_ham_set_kinetic(h, 0) == 0
        buf = ctypes.create_string_buffer(8 * 512)
        assert lib.qsb_ham_apply_host(h, 0, 0, 1, buf, buf, d(0), d(0), d(0), 0, None) == 4   # no potential
        assert b"potential" in lib.qsb_last_error()
        assert lib.qsb_ham_apply_host(h, 0, 0, 1, None, buf, d(0), d(0), d(0), 0, None) == 1  # null psi
    finally:
        assert lib.qsb_ham_destroy(h) == 0
    pos = (ctypes.c_double * 3)(0, 0, 0)
    q = (ctypes.c_double * 1)(1.0)
    bad_cell = (ctypes.c_double * 3)(5.0, 0.0, 5.0)
    e = ctypes.c_double()
    assert lib.qsb_ewald(1, pos, q, bad_cell, ctypes.byref(e), None) == 1 and b"cell" in lib.qsb_last_error()
    assert lib.qsb_relax_lbfgs(None, 1, pos, None, 1, None, None, None, d(9.0), None, None, None, None, None,
                               None, None, 4, 10, d(1e-8), 10, d(1e-4), d(0.2), 5, None, None, None, None) == 1
