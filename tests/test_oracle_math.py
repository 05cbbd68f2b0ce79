"""The oracle's own FFT and quadrature against independent references (CPU).

FFTW and GSL are not in the reference tree; the oracle restates their
contracts (unnormalised DFT with sign -1 forward; QUADPACK 21-point
Gauss-Kronrod).  These tests pin the restatements against numpy's pocketfft,
direct DFT sums, scipy's QUADPACK and exact polynomial integrals.
"""

import ctypes as C

import numpy as np
import pytest

import oracle.pyoracle as po


def _lib():
    lib = po._load()
    lib.offt_c2c_1d.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.offt_c2c_3d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.offt_r2c_3d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.offt_c2r_3d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.oq_qk21.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double] + [C.POINTER(C.c_double)] * 4
    lib.oq_qags.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return lib


@pytest.mark.parametrize("n", [8, 12, 16, 24, 48, 96, 100, 128, 7 * 5 * 3])
def test_fft1d_vs_direct_dft(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.exp(-2j * np.pi * np.outer(np.arange(n), np.arange(n)) / n) @ x
    y = x.copy()
    _lib().offt_c2c_1d(y.ctypes.data, n, -1)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    _lib().offt_c2c_1d(y.ctypes.data, n, +1)
    assert np.abs(y / n - x).max() <= 1e-13 * np.abs(x).max()


@pytest.mark.parametrize("n", [16, 48, 64])
def test_fft3d_vs_numpy(n):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    y = x.copy()
    _lib().offt_c2c_3d(y.ctypes.data, n, n, n, -1)
    ref = np.fft.fftn(x)
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    _lib().offt_c2c_3d(y.ctypes.data, n, n, n, +1)
    assert np.abs(y - n**3 * x).max() <= 1e-12 * n**3 * np.abs(x).max()


@pytest.mark.parametrize("n", [16, 48])
def test_r2c_c2r_padded_layout(n):
    """fftw_mpi r2c/c2r layouts: padded real [n][n][2(n/2+1)], half complex."""
    rng = np.random.default_rng(5)
    p = 2 * (n // 2 + 1)
    real = rng.standard_normal((n, n, n))
    padded = np.zeros((n, n, p))
    padded[:, :, :n] = real
    half = np.empty((n, n, n // 2 + 1), dtype=np.complex128)
    _lib().offt_r2c_3d(padded.ctypes.data, half.ctypes.data, n, n, n, p)
    ref = np.fft.rfftn(real)
    assert np.abs(half - ref).max() <= 1e-12 * np.abs(ref).max()
    out = np.zeros((n, n, p))
    _lib().offt_c2r_3d(half.ctypes.data, out.ctypes.data, n, n, n, p)
    assert np.abs(out[:, :, :n] / n**3 - real).max() <= 1e-13 * np.abs(real).max()


def test_gk21_exact_for_polynomials():
    """21-point Kronrod is exact to degree 31, so the table is right."""
    lib = _lib()
    F = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
    for deg in (0, 5, 17, 31):
        f = F(lambda x, p, d=deg: x**d)
        r, e, ra, rs = (C.c_double() for _ in range(4))
        lib.oq_qk21(f, None, -1.0, 1.0, C.byref(r), C.byref(e), C.byref(ra), C.byref(rs))
        exact = (1 - (-1) ** (deg + 1)) / (deg + 1)
        assert abs(r.value - exact) <= 1e-14


def test_scale_factor_integrals_vs_scipy():
    """dt = int da / (H a^n) as Timestep_criteria integrates it
    (src/CosmoBEC_MPI.cpp:66-68; integrands src/struct3D.h:127-146)."""
    from scipy.integrate import quad

    lib = _lib()
    cst = po.oracle_constants()
    H0, Om = cst["H_0"], cst["Omega_m0"]
    F = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
    for n in (2, 3, 4):
        f = F(lambda x, p, n=n: 1.0 / (H0 * np.sqrt(Om / x**3 + 1 - Om) * x**n))
        for a, da in ((1 / 51, 1e-3), (0.05, 0.02), (0.3, 0.2)):
            r, e = C.c_double(), C.c_double()
            lib.oq_qags(f, None, a, a + da, 0.0, 1e-10, 1000, C.byref(r), C.byref(e))
            ref, _ = quad(lambda x: 1.0 / (H0 * np.sqrt(Om / x**3 + 1 - Om) * x**n), a, a + da, epsabs=0,
                          epsrel=1e-13)
            assert r.value == pytest.approx(ref, rel=1e-12)
