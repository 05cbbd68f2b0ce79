"""Host-side helpers of the benchmark (no GPU): step scale, self-interaction
strength, profiled traffic lookup."""

import importlib.util
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _a_after(bench, N, C, nsteps):
    m2Mpc, s2Myr = 3.086e22, 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    hbar = 6.58211928e-16 / s2Myr
    c = 2.99792458e8 / m2Mpc * s2Myr
    H0, Om = 0.677 * 100 * s2Myr / m2Mpc * 1e3, 0.276
    dx = 2.0 * (bench.XMAX / 0.677) / N
    A = 4.0 / (3.0 * math.pi) * (bench.MFDM / c**2) / hbar * dx**2
    a = bench.A0
    for _ in range(nsteps):
        a += H0 * math.sqrt(Om / a**3 + 1 - Om) * a * C * A * a * a
    return a


@pytest.mark.parametrize("N,nsteps", [(64, 100), (128, 200), (512, 1000)])
def test_step_scale_reaches_half(bench, N, nsteps):
    C = bench.dt_scale_for(N, nsteps)
    assert _a_after(bench, N, C, nsteps) == pytest.approx(0.5, rel=1e-6)


def test_step_scale_of_the_benchmark(bench):
    # the scale quoted for 512^3 / 1000 steps
    assert bench.dt_scale_for(512, 1000) == pytest.approx(0.6957, abs=1e-4)


def test_g_is_linear_in_the_phase_and_scales_with_the_density(bench):
    rng = np.random.default_rng(0)
    psi = (1.0 + 0.1 * rng.standard_normal((8, 8, 8))) * 1e50 + 0j
    C = bench.dt_scale_for(64, 100)
    g1 = bench.g_for_phase(64, psi, C, 0.01)
    g2 = bench.g_for_phase(64, psi, C, 0.02)
    assert g1 > 0 and g2 == pytest.approx(2 * g1, rel=1e-12)
    assert bench.g_for_phase(64, 2 * psi, C, 0.01) == pytest.approx(g1 / 4, rel=1e-12)
    assert bench.g_for_phase(64, psi, C, 0.0) == 0.0


def test_profiled_traffic_lookup(bench):
    t = bench.profiled_traffic("fp32", "P5_ifft_z_density_r2c_z", 512)
    assert t is not None and 1e9 < t < 1e10
    assert bench.profiled_traffic("fp32", "P5_ifft_z_density_r2c_z", 256) is None
    t64 = bench.profiled_traffic("fp64", "P5_ifft_z_density_r2c_z", 512)
    assert t64 is not None and 1.5 * t < t64 < 2.5 * t  # FP64 moves twice the bytes
    assert bench.profiled_traffic("fp64", "P5_ifft_z_density_r2c_z", 1024) is None
