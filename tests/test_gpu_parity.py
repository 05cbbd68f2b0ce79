"""GPU path against the reference and the oracle (needs a B200).

* native runs through the C ABI against the files the reference's own code
  wrote (tests/golden): same snapshot names, headers, and psi within 1e-10
  relative L2 (the FP64 bar); voutput.dat bit-identical;
* the BECMPI executable against the same files;
* fixed-step mode at 64^3 / 100 steps against the oracle (FP64, 1e-10);
* the stand-alone 3-D FFT against numpy;
* FP32-mixed against FP64;
* invariants (norm conservation, free-particle plane wave) and error paths.
"""

import os
import shutil
import subprocess

import numpy as np
import pytest

import ifdm_code_b200 as ifdm
from ifdm_code_b200 import IfdmError, Simulation
from ifdm_code_b200.synthetic_ic import make_ic
from oracle import Oracle, OracleArgs
from tests.snapshot_util import compare_dirs, read_snapshot, rel_l2

pytestmark = pytest.mark.gpu

PSI_TOL = 1e-10  # FP64 drop-in bar: relative L2 on psi


def _sim_from_manifest(m, out, golden_dir, **kw):
    a = m["args"]
    return Simulation(mfdm=float(a[0]), g=float(a[1]), xmax=float(a[2]), res=int(a[3]), t_write=int(a[4]),
                      t_stop=int(a[5]), ti=int(a[6]), opath=out, icpath=os.path.join(golden_dir, m.get("ic", "")),
                      **kw)


@pytest.mark.parametrize("case,stan", [("ref16", False), ("ref16_stan", True), ("ref16_g", False),
                                       ("ref32", False)])
def test_native_run_matches_reference(tmp_path, golden_dir, manifest, case, stan):
    m = manifest[case]
    out = str(tmp_path) + "/"
    with _sim_from_manifest(m, out, golden_dir, stan=stan) as s:
        s.load_ic()
        s.run()
    N = int(m["args"][3])
    if case == "ref32":  # the fixture keeps three of the snapshots
        for f in os.listdir(out):
            if f.endswith(".dat") and f not in m["files"]:
                os.remove(os.path.join(out, f))
    worst = compare_dirs(out, os.path.join(golden_dir, case), m["files"], N, PSI_TOL)
    assert worst <= PSI_TOL
    assert open(os.path.join(out, "voutput.dat"), "rb").read() == open(
        os.path.join(golden_dir, case, "voutput.dat"), "rb").read()


def test_rerun_matches_reference(tmp_path, golden_dir, manifest):
    m = manifest["ref16_rerun"]
    a = m["args"]
    out = str(tmp_path) + "/"
    with Simulation(mfdm=float(a[0]), g=float(a[1]), xmax=float(a[2]), res=int(a[3]), t_write=int(a[4]),
                    t_stop=int(a[5]), ti=int(a[6]), opath=out, icpath=os.path.join(golden_dir, "ref16") + "/",
                    rerun=1) as s:
        s.load_snapshot(int(a[6]))
        s.run()
    compare_dirs(out, os.path.join(golden_dir, "ref16_rerun"), m["files"], 16, PSI_TOL)


def test_cli_matches_reference(tmp_path, golden_dir, manifest):
    m = manifest["ref16"]
    args = list(m["args"])
    args[7] = str(tmp_path) + "/"
    args[8] = os.path.join(golden_dir, m["ic"])
    r = subprocess.run([ifdm.BIN_PATH] + args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    compare_dirs(str(tmp_path), os.path.join(golden_dir, "ref16"), m["files"], 16, PSI_TOL)
    ref_lines = open(os.path.join(golden_dir, "ref16", "stdout.txt")).read()
    assert ref_lines.count(" tn = ") == r.stdout.count(" tn = ")


@pytest.fixture(scope="module")
def ic64(tmp_path_factory):
    d = tmp_path_factory.mktemp("ic64")
    make_ic(str(d / "ic"), 64, seed=0)
    return str(d / "ic")


def test_fixed_steps_64_vs_oracle(ic64, tmp_path):
    """64^3, 100 fixed-mode steps from z = 50: FP64 GPU vs the oracle."""
    C = 0.111
    o = Oracle(OracleArgs(res=64, opath=str(tmp_path) + "/", icpath=ic64))
    o.load_ic()
    psi0 = o.psi()
    o.run_fixed(100, C)
    ref = o.psi()
    with Simulation(2.5e-24, 0.0, 5.0, 64, opath=str(tmp_path) + "/", icpath=ic64) as s:
        s.load_ic()
        assert rel_l2(s.get_psi(), psi0) <= 1e-12
        s.step(100, C)
        got = s.get_psi()
        st = s.state()
    assert st["steps"] == 100 and st["a"] == pytest.approx(o.a, rel=1e-12)
    assert rel_l2(got, ref) <= PSI_TOL


def test_fixed_steps_self_interaction_vs_oracle(ic64, tmp_path):
    g = 1e-62
    o = Oracle(OracleArgs(res=64, g=g, opath=str(tmp_path) + "/", icpath=ic64))
    o.load_ic()
    o.run_fixed(40, 0.3)
    with Simulation(2.5e-24, g, 5.0, 64, opath=str(tmp_path) + "/", icpath=ic64) as s:
        s.load_ic()
        s.step(40, 0.3)
        assert rel_l2(s.get_psi(), o.psi()) <= PSI_TOL
        assert s.state()["a"] == pytest.approx(o.a, rel=1e-12)


def test_phi_matches_oracle(ic64, tmp_path):
    o = Oracle(OracleArgs(res=64, opath=str(tmp_path) + "/", icpath=ic64))
    o.load_ic()
    o.poisson()
    with Simulation(2.5e-24, 0.0, 5.0, 64, opath=str(tmp_path) + "/", icpath=ic64) as s:
        s.load_ic()
        phi = s.get_phi()
    assert rel_l2(phi, o.phi()) <= 1e-12


@pytest.mark.parametrize("n", [16, 32, 48, 64, 96, 128, 256])
def test_fft3d_matches_numpy(n):
    import torch

    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    ref = np.fft.fftn(x)
    for dt, tol, comp in ((torch.complex128, 1e-13, None), (torch.complex64, 2e-6, None),
                          (torch.complex64, 2e-7, "fp64")):
        t = torch.from_numpy(x).to(dt).cuda()
        ifdm.fft3d_(t, -1, comp)
        torch.cuda.synchronize()
        got = t.cpu().numpy()
        assert rel_l2(got, ref) <= tol, (n, dt, comp)
        ifdm.fft3d_(t, +1, comp)
        torch.cuda.synchronize()
        assert rel_l2(t.cpu().numpy() / n**3, x) <= tol


@pytest.mark.parametrize("prec,tol", [("fp32", 3e-5), ("mixed", 2e-6)])
def test_reduced_precision_close_to_fp64(ic64, tmp_path, prec, tol):
    """64^3, 100 steps: density relative L2 against the FP64 path.  FP32
    arithmetic stays within 3e-5; FP64 arithmetic with stochastically rounded
    FP32 storage within 2e-6."""
    dens = {}
    for p in ("fp64", prec):
        with Simulation(2.5e-24, 0.0, 5.0, 64, opath=str(tmp_path) + "/", icpath=ic64, precision=p) as s:
            s.load_ic()
            s.step(100, 0.111)
            dens[p] = np.abs(s.get_psi()) ** 2
    assert rel_l2(dens[prec], dens["fp64"]) <= tol


def test_norm_conserved_and_plane_wave(tmp_path):
    """Kick and drift are unitary; with phi = 0 (uniform |psi|) and g = 0 a
    plane wave only gains exp(-i hbar c^2 k^2/(2m) dt_KE)."""
    N = 32
    xmax = 5.0 / 0.677
    x = xmax / N - xmax + np.arange(N) * (2 * xmax / N)
    kx = 3 * np.pi / xmax
    psi = np.exp(1j * kx * x)[:, None, None] * np.ones((N, N, N)) * 1e50
    with Simulation(2.5e-24, 0.0, 5.0, N, opath=str(tmp_path) + "/") as s:
        s.set_psi(psi, 0.05)
        s.step(3, 1.0)
        got = s.get_psi()
        st = s.state()
    assert np.sum(np.abs(got) ** 2) == pytest.approx(np.sum(np.abs(psi) ** 2), rel=1e-12)
    # total drift phase over the three steps equals the sum of per-step phases;
    # compare the relative phase pattern instead: psi/psi0 must be uniform
    ratio = got / psi
    assert np.abs(ratio - ratio.flat[0]).max() <= 1e-10
    assert st["steps"] == 3


def test_error_paths(tmp_path, golden_dir):
    with pytest.raises(IfdmError, match="UNSUPPORTED"):
        Simulation(2.5e-24, 0.0, 5.0, 20)
    with Simulation(2.5e-24, 0.0, 5.0, 16, opath=str(tmp_path) + "/", icpath=str(tmp_path / "nope")) as s:
        with pytest.raises(IfdmError, match="IO"):
            s.load_ic()
        with pytest.raises(IfdmError, match="STATE"):
            s.step(1)
    # IC box 10 Mpc/h against xmax 4 Mpc/h
    with Simulation(2.5e-24, 0.0, 4.0, 16, opath=str(tmp_path) + "/",
                    icpath=os.path.join(golden_dir, "ic16_s1")) as s:
        with pytest.raises(IfdmError, match="BOXSIZE"):
            s.load_ic()
    # truncated snapshot
    src = os.path.join(golden_dir, "ref16", "output1.dat")
    d = tmp_path / "trunc"
    d.mkdir()
    with open(src, "rb") as f:
        raw = f.read()
    (d / "output1.dat").write_bytes(raw[: len(raw) // 2])
    with Simulation(2.5e-24, 0.0, 5.0, 16, opath=str(tmp_path) + "/", icpath=str(d) + "/", rerun=1) as s:
        with pytest.raises(IfdmError, match="IO"):
            s.load_snapshot(1)


@pytest.fixture(scope="module")
def ic128(tmp_path_factory):
    d = tmp_path_factory.mktemp("ic128")
    make_ic(str(d / "ic"), 128, seed=5)
    return str(d / "ic")


def test_fixed_steps_128_vs_oracle(ic128, tmp_path):
    """128^3 runs the TMA-pipelined y/x passes: FP64 against the oracle."""
    o = Oracle(OracleArgs(res=128, opath=str(tmp_path) + "/", icpath=ic128))
    o.load_ic()
    o.run_fixed(20, 0.22)
    with Simulation(2.5e-24, 0.0, 5.0, 128, opath=str(tmp_path) + "/", icpath=ic128) as s:
        s.load_ic()
        s.step(20, 0.22)
        assert rel_l2(s.get_psi(), o.psi()) <= PSI_TOL
        assert s.state()["device_error"] == 0


@pytest.mark.parametrize("prec", ["fp32", "fp64", "mixed"])
def test_tma_passes_match_plain_passes(ic128, tmp_path, prec, monkeypatch):
    """The TMA pipeline computes the same transform as the plain passes (equal
    up to floating-point contraction differences between the two kernels)."""
    out = {}
    for tma in (True, False):
        if tma:
            monkeypatch.delenv("IFDM_NO_TMA", raising=False)
        else:
            monkeypatch.setenv("IFDM_NO_TMA", "1")
        with Simulation(2.5e-24, 0.0, 5.0, 128, opath=str(tmp_path) + "/", icpath=ic128, precision=prec) as s:
            s.load_ic()
            s.step(5, 0.22)
            out[tma] = s.get_psi()
    assert rel_l2(out[True], out[False]) <= (1e-13 if prec == "fp64" else 2e-6)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_bulk_copy_z_passes_match_plain_passes_256(prec, monkeypatch):
    """At 256^3 the z passes run the bulk-copy kernels (FP64 with 4-row tiles,
    FP32 with 8-row tiles) and the y/x passes the TMA kernels; three fixed
    steps against the plain kernels from the same psi.  In FP32 the TMA x
    pass forms the drift in FP64 and the plain one in FP32, and phi comes
    from the density fluctuation |psi|^2 - mu, which magnifies relative
    differences of psi (phi measured 2.8e-6 apart)."""
    import bench
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    N = 256
    psi0 = zeldovich_psi(N, xmax=bench.XMAX, seed=0, a=bench.A0, mfdm=bench.MFDM)
    C = bench.dt_scale_for(N)
    g = bench.g_for_phase(N, psi0, C, 0.1)
    out = {}
    for tma in (True, False):
        if tma:
            monkeypatch.delenv("IFDM_NO_TMA", raising=False)
        else:
            monkeypatch.setenv("IFDM_NO_TMA", "1")
        with Simulation(bench.MFDM, g, bench.XMAX, N, precision=prec) as s:
            s.set_psi(psi0, bench.A0)
            s.step(3, C)
            out[tma] = (s.get_psi(), s.get_phi(), s.state())
    assert out[True][2]["device_error"] == 0
    assert out[True][2]["a"] == out[False][2]["a"]
    tol_psi, tol_phi = (1e-13, 1e-13) if prec == "fp64" else (2e-6, 1e-5)
    assert rel_l2(out[True][0], out[False][0]) <= tol_psi
    assert rel_l2(out[True][1], out[False][1]) <= tol_phi


def test_strong_self_interaction_follows_oracle(tmp_path):
    """The self-interaction strength the 512^3 precision configuration names
    (0.1 rad per step at the densest cell) with its step scale (0.696 of the
    kinetic limit, 1000 steps to a = 0.5), at 128^3 for 30 steps: the FP64
    path follows the oracle to the FP64 bar in the regime where the scheme
    amplifies max|psi|^2, so that growth belongs to the scheme, not to the
    kernels."""
    import bench
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    N, C, steps = 128, 0.696, 30
    psi0 = zeldovich_psi(N, xmax=bench.XMAX, seed=0, a=bench.A0, mfdm=bench.MFDM)
    g = bench.g_for_phase(N, psi0, C, 0.1)
    o = Oracle(OracleArgs(res=N, g=g, opath=str(tmp_path) + "/"))
    o.set_psi(psi0, bench.A0)
    o.run_fixed(steps, C)
    with Simulation(bench.MFDM, g, bench.XMAX, N, opath=str(tmp_path) + "/") as s:
        s.set_psi(psi0, bench.A0)
        s.step(1, C)
        r1 = s.state()["max_rho"]
        s.step(steps - 1, C)
        st = s.state()
        err = rel_l2(s.get_psi(), o.psi())
    print(f"128^3, 0.1 rad/step, C={C}: max|psi|^2 grew x{st['max_rho'] / r1:.3f} over {steps} steps; "
          f"psi rel L2 vs oracle {err:.3e}")
    assert st["a"] == pytest.approx(o.a, rel=1e-12)
    assert err <= PSI_TOL
