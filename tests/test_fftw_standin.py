"""CPU checks of the FFTW 3 stand-in (oracle/ref_shim/fftw_dft.cpp) that the
reference's FFT code runs on in oracle/_ref/libqsref_fft.so: FFTW's documented
transforms (unnormalised, sign -1 forward / +1 backward, row-major, the
advanced-interface strides and distances, half-spectrum r2c / c2r) against
numpy's FFT of the same definition."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_fft_available(), reason="reference FFT oracle library not built here")

FORWARD, BACKWARD, ESTIMATE = -1, 1, 1 << 6


def _lib():
    lib = ctypes.CDLL(O.LIB_REF_FFT)
    vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
    lib.fftw_plan_many_dft.restype = vp
    lib.fftw_plan_many_dft.argtypes = [ctypes.c_int, ip, ctypes.c_int, vp, ip, ctypes.c_int, ctypes.c_int, vp, ip,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint]
    lib.fftw_plan_dft_3d.restype = vp
    lib.fftw_plan_dft_3d.argtypes = [ctypes.c_int] * 3 + [vp, vp, ctypes.c_int, ctypes.c_uint]
    lib.fftw_plan_dft_r2c_3d.restype = vp
    lib.fftw_plan_dft_r2c_3d.argtypes = [ctypes.c_int] * 3 + [vp, vp, ctypes.c_uint]
    lib.fftw_plan_dft_c2r_3d.restype = vp
    lib.fftw_plan_dft_c2r_3d.argtypes = [ctypes.c_int] * 3 + [vp, vp, ctypes.c_uint]
    for f in ("fftw_execute", "fftw_destroy_plan"):
        getattr(lib, f).argtypes = [vp]
    lib.fftw_execute_dft.argtypes = [vp, vp, vp]
    return lib


def _c(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("shape,sign", [((6, 5, 8), FORWARD), ((9, 4, 7), BACKWARD), ((1, 12, 3), FORWARD)])
def test_3d_in_place(shape, sign):
    lib = _lib()
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    want = np.fft.fftn(a) if sign == FORWARD else np.fft.ifftn(a) * a.size
    buf = np.ascontiguousarray(a, np.complex128)
    p = lib.fftw_plan_dft_3d(*shape, _c(buf), _c(buf), sign, ESTIMATE)
    lib.fftw_execute(p)
    lib.fftw_destroy_plan(p)
    assert np.abs(buf - want).max() <= 1e-13 * np.abs(want).max()


def test_many_with_stride_and_distance():
    # the layout of FFTW_ExecutorMany3D: howmany transforms of n (z, y, x), stride 1, distance ld > n
    lib = _lib()
    rng = np.random.default_rng(2)
    n = np.array([5, 6, 4], np.int32)
    size, ld, howmany = int(np.prod(n)), int(np.prod(n)) + 7, 3
    buf = np.zeros(howmany * ld, np.complex128)
    a = rng.standard_normal((howmany, *n)) + 1j * rng.standard_normal((howmany, *n))
    for b in range(howmany):
        buf[b * ld:b * ld + size] = a[b].ravel()
    pad = buf.copy()
    ip = n.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    p = lib.fftw_plan_many_dft(3, ip, howmany, _c(buf), ip, 1, ld, _c(buf), ip, 1, ld, FORWARD, ESTIMATE)
    lib.fftw_execute_dft(p, _c(buf), _c(buf))
    lib.fftw_destroy_plan(p)
    for b in range(howmany):
        want = np.fft.fftn(a[b]).ravel()
        got = buf[b * ld:b * ld + size]
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        np.testing.assert_array_equal(buf[b * ld + size:(b + 1) * ld], pad[b * ld + size:(b + 1) * ld])


def test_r2c_and_c2r():
    lib = _lib()
    rng = np.random.default_rng(3)
    shape = (6, 5, 8)
    x = np.ascontiguousarray(rng.standard_normal(shape))
    half = np.zeros((6, 5, 5), np.complex128)
    p = lib.fftw_plan_dft_r2c_3d(*shape, _c(x), _c(half), ESTIMATE)
    lib.fftw_execute(p)
    lib.fftw_destroy_plan(p)
    want = np.fft.rfftn(x)
    assert np.abs(half - want).max() <= 1e-13 * np.abs(want).max()
    back = np.zeros(shape)
    p = lib.fftw_plan_dft_c2r_3d(*shape, _c(half), _c(back), ESTIMATE)
    lib.fftw_execute(p)
    lib.fftw_destroy_plan(p)
    assert np.abs(back / x.size - x).max() <= 1e-13 * np.abs(x).max()
