"""The reference's production grid, 1024^3 (job.sh:24), on one B200 (needs a B200).

* the stand-alone 3-D FFT at n = 1024 (the 4 x 8 x 8 x 4 plan, 16 elements per
  thread in the plain passes) against cuFFT through torch.fft, complex128 and
  complex64, compared on the device;
* two leap-frog steps of a 1024^3 box in FP64 through the TMA passes against
  the plain passes, and the FP32 path against FP64 (density and psi);
* the mixed mode is not compiled at this size and says so.

Device memory: up to ~110 GB at a time (psi, phi and the half spectrum of an
FP64 box are 34 GB); host memory stays small (fields stay on the device).
"""

import numpy as np
import pytest

import ifdm_code_b200 as ifdm
from ifdm_code_b200 import IfdmError, Simulation

pytestmark = pytest.mark.gpu

N = 1024
MFDM, XMAX, A0 = 2.5e-24, 5.0, 1.0 / 51.0


def _rel(a, b):
    return float((a - b).abs().norm() / b.abs().norm())


def test_fft3d_1024_matches_cufft():
    import torch

    gen = torch.Generator(device="cuda")
    gen.manual_seed(1024)
    for dt, tol in ((torch.complex128, 1e-13), (torch.complex64, 3e-6)):
        x = torch.randn((N, N, N), generator=gen, device="cuda", dtype=dt)
        ref = torch.fft.fftn(x)
        t = x.clone()
        ifdm.fft3d_(t, -1)
        torch.cuda.synchronize()
        err = _rel(t, ref)
        del ref
        assert err <= tol, (dt, err)
        ifdm.fft3d_(t, +1)
        torch.cuda.synchronize()
        err = _rel(t / N**3, x)
        assert err <= tol, (dt, err)
        del x, t
        torch.cuda.empty_cache()


def test_mixed_1024_unsupported():
    assert not ifdm.supported_res(N, "mixed") and ifdm.supported_res(N, "fp32") and ifdm.supported_res(N, "fp64")
    with pytest.raises(IfdmError, match="UNSUPPORTED"):
        Simulation(MFDM, 0.0, XMAX, N, precision="mixed")


def test_steps_1024(monkeypatch):
    """FP64 TMA passes equal the plain passes to rounding; FP32 follows FP64."""
    import bench
    import torch
    from ifdm_code_b200.synthetic_ic import zeldovich_psi_device

    C = bench.dt_scale_for(N)
    psi0 = zeldovich_psi_device(N, xmax=XMAX, seed=3, a=A0, mfdm=MFDM)
    torch.cuda.synchronize()  # psi0 is read on the library's own stream
    out = {}
    for name, prec, tma in (("fp64", "fp64", True), ("fp64_plain", "fp64", False), ("fp32", "fp32", True)):
        if tma:
            monkeypatch.delenv("IFDM_NO_TMA", raising=False)
        else:
            monkeypatch.setenv("IFDM_NO_TMA", "1")
        with Simulation(MFDM, 0.0, XMAX, N, precision=prec) as s:
            s.set_psi(psi0, A0)
            s.step(2, C)
            st = s.state()
            assert st["device_error"] == 0 and st["steps"] == 2
            res = torch.empty_like(psi0)
            s.get_psi_into(res)
            out[name] = res
        torch.cuda.empty_cache()
    e_tma = _rel(out["fp64"], out["fp64_plain"])
    e32 = _rel(out["fp32"], out["fp64"])
    d32 = _rel(out["fp32"].abs() ** 2, out["fp64"].abs() ** 2)
    print(f"1024^3, 2 steps: fp64 tma vs plain {e_tma:.2e}; fp32 vs fp64 psi {e32:.2e}, density {d32:.2e}")
    assert e_tma <= 1e-13
    assert e32 <= 1e-6 and d32 <= 1e-6  # measured: 8.0e-8, 1.1e-7 (TMA vs plain 8.9e-17)
