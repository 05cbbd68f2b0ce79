#!/usr/bin/env python
"""Benchmark: cell-steps/s of the leap-frog Schroedinger-Poisson step at 512^3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (ours): one 512^3 box (xmax = 5 Mpc/h, mfdm = 2.5e-24 eV, g = 0) from a
seeded z = 50 Zel'dovich field, fixed-step mode with the reference's timestep
rule scaled so 1000 steps reach a = 0.5.  A "step" is one full leap-frog step
(timestep + kick + FFT + drift + iFFT + Poisson + kick, 10 kernels).  The
headline `value` is the fastest path (FP32, mixed or FP64) whose density stays
within 1e-5 of FP64 after 1000 steps, with psi resident in HBM; every path is
timed the same way beside it.  `e2e` times the public API
with host buffers: psi uploaded from pinned memory, K steps, psi read back.
With --gpus N > 1 (torchrun) every rank advances its own box (replicas: one
box per GPU, no exchange between them), timed as the max over ranks.

--impl reference times the reference's own CPU code (oracle/_ref/BECMPI_ref,
its unmodified sources with single-rank MPI/FFTW/GSL shims) on this host:
rerun from a synthetic 512^3 snapshot, per-step time from the shim's
timestamps at the two MPI_Allreduce calls of each step.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 512
XMAX = 5.0
MFDM = 2.5e-24
A0 = 1.0 / 51.0
METRIC = "cell-steps/s at 512^3, FP32-mixed vs FP64 at <=1e-5 density err; adjoint/fwd"


def dt_scale_for(N: int, nsteps: int = 1000, a_end: float = 0.5, xmax: float = XMAX, mfdm: float = MFDM) -> float:
    """Multiplier C of the reference's kinetic timestep rule
    (src/CosmoBEC_MPI.cpp:32) so that nsteps kinetic-limited steps take a from
    1/51 to a_end."""
    import math

    m2Mpc, s2Myr = 3.086e22, 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    hbar = 6.58211928e-16 / s2Myr
    c = 2.99792458e8 / m2Mpc * s2Myr
    H0 = 0.677 * 100 * s2Myr / m2Mpc * 1e3
    Om = 0.276
    dx = 2.0 * (xmax / 0.677) / N
    A = 4.0 / (3.0 * math.pi) * (mfdm / c**2) / hbar * dx**2

    def a_after(C):
        a = A0
        for _ in range(nsteps):
            a += H0 * math.sqrt(Om / a**3 + 1 - Om) * a * C * A * a * a
            if a > 10:
                break
        return a

    lo, hi = 1e-6, 100.0
    for _ in range(200):
        mid = math.sqrt(lo * hi)
        if a_after(mid) > a_end:
            hi = mid
        else:
            lo = mid
    return math.sqrt(lo * hi)


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[0]) for r in self.rows if num(r[0])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(self.rows[0][1]),
                "reasons": reasons, "samples": len(self.rows),
                "power_w_max": max((num(r[2]) or 0.0) for r in self.rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def time_steps(sim, steps: int, warmup: int, dt_scale: float, torch):
    """Device time of `steps` fixed-mode steps on the library's stream."""
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.step(warmup, dt_scale)
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps, dt_scale)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def g_for_phase(N: int, psi0, dt_scale: float, phase: float) -> float:
    """Self-interaction g [eV cm^3] whose kick turns the densest cell of psi0 by
    `phase` radians in the first step: that turn is dt_QI (g/hbar) max|psi|^2
    with dt_QI = integral of da/(H a^4) over the first, kinetic-limited step
    (src/CosmoBEC_MPI.cpp:30-68, src/struct3D.h:127-146), linear in g."""
    import math

    import numpy as np
    from scipy.integrate import quad

    if phase <= 0:
        return 0.0
    m2Mpc, cm2Mpc, s2Myr = 3.086e22, 3.086e24, 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    hbar = 6.58211928e-16 / s2Myr
    c = 2.99792458e8 / m2Mpc * s2Myr
    H0, Om = 0.677 * 100 * s2Myr / m2Mpc * 1e3, 0.276
    dx = 2.0 * (XMAX / 0.677) / N
    dt_ke = 4.0 / (3.0 * math.pi) * (MFDM / c**2) / hbar * dx**2 * A0 * A0

    def H(a):
        return H0 * math.sqrt(Om / a**3 + 1 - Om)

    da = H(A0) * A0 * dt_ke * dt_scale
    dt_qi = quad(lambda a: 1.0 / (H(a) * a**4), A0, A0 + da, epsabs=0, epsrel=1e-12)[0]
    max_rho = float(np.max(np.abs(psi0) ** 2))
    return phase * hbar * cm2Mpc**3 / (dt_qi * max_rho)


def calibrate_g(args) -> None:
    """Print the g of the self-interaction config: the g=0 FP64 run of the
    benchmark (1000 steps to a = 0.5) gives, per step, the turn per unit g of
    the densest cell, dt_QI max|psi|^2 / hbar; g is set so that the largest of
    these over the run is --g-phase radians."""
    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    N = args.res
    C = dt_scale_for(N)
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=0, a=A0, mfdm=MFDM)
    s2Myr = 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    hbar, cm2Mpc = 6.58211928e-16 / s2Myr, 3.086e24
    peak, at = 0.0, 0
    with ifdm.Simulation(MFDM, 0.0, XMAX, N) as sim:
        sim.set_psi(psi0, A0)
        for n in range(args.precision_steps):
            sim.step(1, C)
            st = sim.state()
            per_g = st["dt_QI"] * st["max_rho"] / hbar / cm2Mpc ** 3  # radians per unit g [eV cm^3]
            if per_g > peak:
                peak, at = per_g, n
    print(json.dumps({"res": N, "steps": args.precision_steps, "peak_turn_per_unit_g": peak, "at_step": at,
                      "g_eV_cm3": args.g_phase / peak}))


def precision_report(N: int, g: float, nsteps: int, device: int, seed: int = 0) -> dict:
    """Density after nsteps steps (step scale reaching a = 0.5 at step 1000,
    500... as for the benchmark) in mixed and FP32 against FP64 from the same
    IC: relative L2 of the density, norm drift, P(k) ratio per k-bin."""
    import numpy as np

    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    C = dt_scale_for(N, nsteps)
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=seed, a=A0, mfdm=MFDM)
    rho, pks = {}, {}
    for prec in ("fp64", "mixed", "fp32"):
        with ifdm.Simulation(MFDM, g, XMAX, N, precision=prec, device=device) as sim:
            sim.set_psi(psi0, A0)
            sim.step(nsteps, C)
            rho[prec] = np.abs(sim.get_psi()) ** 2
            pks[prec] = sim.power_spectrum(24)["pk"]  # on the device (ifdm_power_spectrum)
            a_end = sim.state()["a"]
    pk_ref = pks["fp64"]
    out = {"res": N, "g": g, "steps": nsteps, "dt_scale": C, "a_end": a_end}
    for prec in ("mixed", "fp32"):
        r, ref = rho[prec], rho["fp64"]
        ratio = pks[prec] / pk_ref
        out[prec] = {"density_relL2": float(np.linalg.norm(r - ref) / np.linalg.norm(ref)),
                     "norm_drift": float(r.sum() / ref.sum() - 1.0),
                     "pk_ratio_max_dev": float(np.max(np.abs(ratio - 1.0))),
                     "pk_ratio_per_bin": [round(float(x), 9) for x in ratio]}
    return out


def cpu_baseline_port(N: int, psi0, dt_scale: float):
    """The oracle (C restatement, OpenMP on every host core) for one step at N^3."""
    from oracle import Oracle, OracleArgs

    o = Oracle(OracleArgs(res=N, mfdm=MFDM, xmax=XMAX))
    o.set_psi(psi0, A0)
    t = time.perf_counter()
    o.run_fixed(1, dt_scale)
    dt = time.perf_counter() - t
    o.close()
    return {"value": N**3 / dt, "unit": "cell-steps/s", "cores": Oracle.num_threads(), "kind": "port",
            "sample": f"1 leap-frog step of the {N}^3 workload ({dt:.1f} s)"}


def profiled_traffic(prec: str, pass_name: str, N: int):
    """DRAM bytes read + written per launch by the pass's kernel at 512^3, from
    the committed ncu summary (profiles/step_512_dram_per_kernel.md: one pass of
    dram__bytes_read.sum + dram__bytes_write.sum over one step), else None."""
    path = os.path.join(ROOT, "profiles", "step_512_dram_per_kernel.md")
    if N != 512 or not os.path.exists(path):
        return None
    key = pass_name.split("_")[0]
    for line in open(path):
        f = line.split()
        if len(f) == 4 and f[0] == "traffic" and f[1] == prec and f[2] == key:
            return float(f[3])
    return None


def snapshot_section(ifdm, N, prec, psi0, G, C, device, iters):
    """Snapshots while stepping, two schedules: one after every step (the
    reference's production state machine writes output<n>.dat each step
    between a = 0.25 and 0.5, src/CosmoBEC_MPI_stan.cpp) and one every 50
    steps.  Wall time per interval (steps + snapshot), three ways: steps
    only; blocking (gather, copy and write inside the call, as the
    reference's writeall); streamed (staged on the device, copied on a copy
    stream and written by the writer thread beside the next steps).  Every
    snapshot gets a new file name, as in the reference's runs (overwriting
    a 2 GiB file costs its truncation, 0.7 s on the box's disk); the files are
    deleted, and dirty pages synced, outside the timed regions."""
    import shutil
    import tempfile

    fbytes = 16 * N ** 3 + 8 * (N + 3)
    d = tempfile.mkdtemp(prefix="ifdm_snap_")
    try:
        free = shutil.disk_usage(d).free
        if free < (iters + 3) * fbytes:
            return {"skipped": f"{free / 1e9:.1f} GB free in {tempfile.gettempdir()}, "
                               f"need {(iters + 3) * fbytes / 1e9:.1f}"}
        out = {"res": N, "path": prec, "iterations": iters, "file_bytes": fbytes, "schedules": {}}
        for every in (1, 50):
            ms = {}
            for mode in ("steps_only", "blocking", "streamed"):
                sim = ifdm.Simulation(MFDM, G, XMAX, N, precision=prec, device=device, opath=d + "/")
                sim.set_psi(psi0, A0)
                sim.step(2, C)
                sim.set_snapshot_streaming(mode == "streamed")
                if mode != "steps_only":  # first use allocates the staging and pinned buffers
                    sim.write_snapshot(9)
                sim.synchronize()
                os.sync()
                t0 = time.perf_counter()
                for i in range(iters):
                    sim.step(every, C)
                    if mode == "blocking":
                        sim.write_snapshot(10 + i)
                    elif mode == "streamed":
                        sim.write_snapshot_async(10 + i)
                sim.flush_snapshots()
                sim.synchronize()
                ms[mode] = (time.perf_counter() - t0) / iters * 1e3
                sim.close()
                for f in os.listdir(d):
                    os.remove(os.path.join(d, f))
            out["schedules"][f"every_{every}_steps"] = {
                "ms_per_interval": {k: round(v, 3) for k, v in ms.items()},
                "snapshot_cost_ms": {k: round(ms[k] - ms["steps_only"], 3) for k in ("blocking", "streamed")},
                "blocking_over_streamed": round(ms["blocking"] / ms["streamed"], 3)}
        out["note"] = ("wall clock around iters x (steps + snapshot), the last file flushed inside the timed "
                       "region; buffered writes to the box's scratch disk")
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def ic_section(ifdm, N, device, cpu_res):
    """Gadget IC pre-processing (src/gadget_IC.h:259-672) at N^3 particles:
    four chunk files written to a scratch folder, then ifdm_load_ic timed
    (files read side by side and streamed to the device, device CIC by a
    stable radix sort by cell, divergence, spectral phase, psi), first call
    and a repeat.  Size-independent check: the deposited mass equals the
    particles' mass (ghost copies and the zero particle of each chunk
    included, as one reference rank deposits them).  The oracle's IC on the
    host cores at cpu_res^3 particles, per particle, stands beside it."""
    import shutil
    import tempfile

    import numpy as np
    import torch

    from ifdm_code_b200.synthetic_ic import write_gadget_chunks, zeldovich_particles_device

    d = tempfile.mkdtemp(prefix="ifdm_ic_")
    try:
        need = 28 * N ** 3 * 1.1
        if shutil.disk_usage(d).free < need:
            return {"skipped": f"{shutil.disk_usage(d).free / 1e9:.1f} GB free, need {need / 1e9:.1f}"}
        t0 = time.perf_counter()
        pos, vel, mass, a, box = zeldovich_particles_device(N, xmax=XMAX, seed=7, device=device)
        torch.cuda.empty_cache()
        write_gadget_chunks(d + "/ic", pos, vel, mass, a, box)
        t_make = time.perf_counter() - t0
        # slots one reference rank deposits: per chunk its particles, the
        # trailing ones beyond the last cell centre again, and one zero particle
        m = N ** 3 // 4
        xg_last = (N - 1) * (box / N) + 0.5 * (box / N)
        slots = 0
        for c in range(4):
            x = pos[c * m:(c + 1) * m, 0].astype(np.float64)
            beyond = x[1:][::-1] > xg_last
            lg = int(np.argmin(beyond)) if not beyond.all() else beyond.size
            slots += m + lg + 1
        del pos, vel
        times = []
        rho_sum = None
        for rep in range(2):
            with ifdm.Simulation(MFDM, 0.0, XMAX, N, opath=d + "/", icpath=d + "/ic", device=device) as sim:
                sim.synchronize()
                t0 = time.perf_counter()
                sim.load_ic()
                sim.synchronize()
                times.append(time.perf_counter() - t0)
                if rep == 1:
                    psi = torch.empty((N, N, N), dtype=torch.complex128, device=f"cuda:{device}")
                    sim.get_psi_into(psi)
                    rho_sum = float((psi.real ** 2 + psi.imag ** 2).sum())
                    del psi
        # |psi|^2 = 1.225^2 rho h^2 1e9 / m_solar, rho = mass per cell / Lg^3 (Msun h^-1 / (kpc/h)^3)
        consts = {"kg2eV": 1.783e-36, "kg2solar": 1.989e30, "h": 0.677}
        m_solar = MFDM * consts["kg2eV"] / consts["kg2solar"]
        Lg = box / N
        want = 1.225 ** 2 * slots * mass * 1e10 / Lg ** 3 * consts["h"] ** 2 * 1e9 / m_solar
        out = {"res": N, "particles": 4 * m, "particle_slots": slots, "files_gb": 28 * N ** 3 / 1e9,
               "make_files_s": round(t_make, 2), "load_ic_s": round(times[0], 3), "load_ic_repeat_s": round(times[1], 3),
               "particles_per_s": 4 * m / times[1],
               "mass_rel_err": abs(rho_sum / want - 1.0)}
    finally:
        shutil.rmtree(d, ignore_errors=True)
    if cpu_res:
        from oracle import Oracle, OracleArgs
        from ifdm_code_b200.synthetic_ic import make_ic

        d = tempfile.mkdtemp(prefix="ifdm_ic_cpu_")
        try:
            make_ic(d + "/ic", cpu_res, seed=7)
            o = Oracle(OracleArgs(res=cpu_res, mfdm=MFDM, xmax=XMAX, opath=d + "/", icpath=d + "/ic"))
            t0 = time.perf_counter()
            o.load_ic()
            dt = time.perf_counter() - t0
            o.close()
            out["cpu_baseline"] = {"value": cpu_res ** 3 / dt, "unit": "particles/s", "cores": Oracle.num_threads(),
                                   "kind": "port", "sample": f"oracle IC at {cpu_res}^3 particles ({dt:.1f} s)"}
        finally:
            shutil.rmtree(d, ignore_errors=True)
    return out


def run_ours(args):
    import numpy as np
    import torch

    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    from ifdm_code_b200.replicas import Replicas

    rep_ = Replicas("nccl")
    world, rank, local = rep_.world, rep_.rank, rep_.local
    N = args.res
    K, W = args.steps, args.warmup
    C = dt_scale_for(N)
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=rank, a=A0, mfdm=MFDM)
    peaks, peak_kind = measured_peaks()
    hbm = float(peaks["hbm_gbs"])

    barrier = rep_.barrier
    max_over_ranks = rep_.max
    # self-interaction of the 512^3 precision config (radians per step at the densest cell: --g-phase)
    G = g_for_phase(N, psi0, C, args.g_phase)
    turn = None
    if G:
        with ifdm.Simulation(MFDM, G, XMAX, N, device=local) as sim:  # check: the first step's turn
            sim.set_psi(psi0, A0)
            sim.step(1, C)
            st = sim.state()
        s2Myr = 60.0 * 60.0 * 24.0 * 365.0 * 1e6
        turn = st["dt_QI"] * (G / 3.086e24 ** 3) / (6.58211928e-16 / s2Myr) * st["max_rho"]

    res = {}
    for prec in ("fp64", "mixed", "fp32"):
        sim = ifdm.Simulation(MFDM, G, XMAX, N, precision=prec, device=local)
        sim.set_psi(psi0, A0)
        t_w = time.perf_counter()
        sim.step(W, C)
        sim.synchronize()
        per_step = (time.perf_counter() - t_w) / max(W, 1)
        # the clock record spans at least ~1.2 s of the same load: untimed steps
        # of this box before and after the timed ones keep the GPU busy while
        # nvidia-smi samples (the timed region alone may be 0.1 s)
        pad = max(1, min(400, int(0.6 / max(per_step, 1e-4))))
        barrier()
        clk = ClockSampler(local)
        with clk:
            sim.step(pad, C)
            ms = time_steps(sim, K, 0, C, torch)
            sim.step(pad, C)
            sim.synchronize()
        barrier()
        ms = max_over_ranks(ms)
        prof = sim.profile_passes(max(3, min(10, K)), C)
        pb = sim.pass_bytes()
        st = sim.state()
        res[prec] = dict(ms=ms, prof=prof, bytes=pb, state=st, clocks=clk.summary())
        if args.precision_steps > 0:
            # the precision gate: density after `precision_steps` steps from the IC
            sim.set_psi(psi0, A0)
            sim.step(args.precision_steps, C)
            res[prec]["rho"] = np.abs(sim.get_psi()) ** 2
            res[prec]["pk"] = sim.power_spectrum(24)["pk"]  # on the device (ifdm_power_spectrum)
            res[prec]["a_end"] = sim.state()["a"]
        sim.close()
        del sim
        torch.cuda.synchronize()
    prec_report = {}
    if args.precision_steps > 0:
        ref = res["fp64"]["rho"]
        pk_ref = res["fp64"]["pk"]
        for prec in ("mixed", "fp32"):
            rho = res[prec]["rho"]
            pk = res[prec]["pk"]
            prec_report[prec] = {
                "steps": args.precision_steps,
                "density_relL2": float(np.linalg.norm(rho - ref) / np.linalg.norm(ref)),
                "norm_drift": float(rho.sum() / ref.sum() - 1.0),
                "pk_ratio_max_dev": float(np.max(np.abs(pk / pk_ref - 1.0))),
                "pk_ratio_per_bin": [round(float(x), 9) for x in pk / pk_ref],
                "a_end": res[prec]["a_end"],
            }
            del res[prec]["rho"]
        del res["fp64"]["rho"]
    # headline: the fastest path whose density error passes the gate (FP64 is the reference)
    gate = 1e-5
    passing = ["fp64"] + [p for p in ("mixed", "fp32") if prec_report and prec_report[p]["density_relL2"] <= gate]
    head = min(passing, key=lambda p: res[p]["ms"])

    # adjoint / forward time: record K_a steps (checkpoint every 20), then the
    # backward sweep (segment replays + adjoint steps), same path as the headline
    adj = None
    if args.adjoint_steps > 0:
        ka = args.adjoint_steps
        sim = ifdm.Simulation(MFDM, G, XMAX, N, precision=head, device=local)
        sim.set_psi(psi0, A0)
        sim.synchronize()
        t0 = time.perf_counter()
        sim.record_steps(ka, C, 20)
        sim.synchronize()
        t_fwd = time.perf_counter() - t0
        # any cotangent (the cost does not depend on it), resident on the device like the state
        gfin = torch.from_numpy(psi0).to(f"cuda:{local}")
        g0 = torch.empty_like(gfin)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.adjoint(gfin, g0)
        sim.synchronize()
        t_bwd = time.perf_counter() - t0
        sim.close()
        del gfin, g0
        # neither leg copies to or from the host: forward = the recorded steps
        # (checkpoint copies and step log included), backward = segment replays + adjoint steps
        adj = {"path": head, "steps": ka, "checkpoint_every": 20, "forward_s": t_fwd, "backward_s": t_bwd,
               "adjoint_over_forward": t_bwd / t_fwd}

    # the headline path, and mixed (whose boxes equal their one-at-a-time runs bit for bit)
    # cuFFT through torch.fft, a reference point only: one forward + inverse 3-D
    # c2c of psi (a step needs this pair, a real-to-complex pair for the
    # Poisson solve, the kick, the drift and the reductions)
    fft_ref = {}
    for name, dt in (("complex64", torch.complex64), ("complex128", torch.complex128)):
        x = torch.from_numpy(psi0).to(device=f"cuda:{local}", dtype=dt)
        for _ in range(2):
            x = torch.fft.ifftn(torch.fft.fftn(x))
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(5):
            x = torch.fft.ifftn(torch.fft.fftn(x))
        ev1.record()
        torch.cuda.synchronize()
        fft_ref[name + "_fft_pair_ms"] = ev0.elapsed_time(ev1) / 5
        del x
        torch.cuda.empty_cache()

    # the 256^3, g = 0 precision config (1000 steps), reported beside the headline
    prec256 = precision_report(256, 0.0, 1000, local) if (args.precision_steps > 0 and N == 512) else None
    # the 256^3 precision config with the self-interaction strength the 512^3
    # configuration names (0.1 rad per step at the densest cell), at which the
    # scheme is stable at 256^3
    prec256g = None
    if args.precision_steps > 0 and N == 512:
        from ifdm_code_b200.synthetic_ic import zeldovich_psi as _zp
        C256 = dt_scale_for(256)
        g256 = g_for_phase(256, _zp(256, xmax=XMAX, seed=0, a=A0, mfdm=MFDM), C256, 0.1)
        prec256g = precision_report(256, g256, 1000, local)
        prec256g["g_phase_rad"] = 0.1

    batch = {p: run_batch(args, p, local, args.adjoint_steps if p == head else 0)
             for p in dict.fromkeys([head, "mixed"])} if args.batch_steps > 0 else None

    ic = ic_section(ifdm, args.ic_res, local, 128 if not args.no_cpu_baseline else 0) if (
        args.ic_res > 0 and rank == 0) else None

    snaps = snapshot_section(ifdm, N, head, psi0, G, C, local, args.snapshot_steps) if (
        args.snapshot_steps > 0 and rank == 0) else None

    # end to end through the C ABI with host buffers (pinned)
    pin_in = torch.from_numpy(psi0.view(np.float64)).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    sim = ifdm.Simulation(MFDM, G, XMAX, N, precision=head, device=local)
    sim.set_psi(pin_in.numpy().view(np.complex128), A0)
    sim.step(W, C)
    sim.synchronize()
    barrier()
    t0 = time.perf_counter()
    sim.set_psi(pin_in.numpy().view(np.complex128), A0)
    sim.step(K, C)
    sim.get_psi(out=pin_out.numpy().view(np.complex128).reshape(N, N, N))
    e2e_s = time.perf_counter() - t0
    sim.close()
    e2e_s = max_over_ranks(e2e_s)

    cells = float(N) ** 3
    value = world * cells * K / (res[head]["ms"] / 1e3)
    vals = {p: world * cells * K / (res[p]["ms"] / 1e3) for p in res}
    fp64_value = vals["fp64"]
    e2e_value = world * cells * K / e2e_s

    def roofline(r, prec):
        names = list(r["prof"].keys())
        ms = [r["prof"][n] for n in names]
        i = max(range(1, len(ms)), key=lambda j: ms[j])
        achieved = r["bytes"][i] / (ms[i] / 1e3) / 1e9
        step_bytes = sum(r["bytes"])
        return {"bound": "hbm", "kernel": names[i], "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": profiled_traffic(prec, names[i], N),
                "algorithmic_bytes": r["bytes"][i], "peak_kind": peak_kind,
                "step_bytes_per_cell": step_bytes / cells,
                "step_achieved_gbs": round(step_bytes / (sum(ms) / 1e3) / 1e9, 1),
                "passes_ms": {n: round(v, 4) for n, v in zip(names, ms)},
                "passes_frac": {n: round(b / (v / 1e3) / 1e9 / hbm, 3) for n, v, b in zip(names, ms, r["bytes"])
                                if b > 0}}

    out = {
        "metric": METRIC,
        "value": value,
        "unit": "cell-steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": res[head]["ms"] / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"mixed": "f32 storage / f64 arithmetic", "fp32": "f32", "fp64": "f64"}[head],
        "path": head,
        "data": "synthetic",
        "config": {"workload": f"{N}^3 leap-frog step, xmax=5 Mpc/h, mfdm=2.5e-24 eV, g={G:.4e} eV cm^3 "
                               f"({args.g_phase} rad/step at the densest cell), z=50 Zel'dovich IC, "
                               f"fixed-step dt_scale={C:.4f} (1000 steps to a=0.5)",
                   "g_eV_cm3": G, "g_turn_first_step_rad": turn,
                   "res": N, "parallelism": f"replicas x{world}" if world > 1 else "1 box",
                   "l2": "inputs larger than L2 (psi fp32 = %.1f GB)" % (8 * cells / 1e9)},
        "paths": {p: {"value": vals[p], "ms_per_step": res[p]["ms"] / K, "over_fp64": vals[p] / fp64_value,
                      "roofline": roofline(res[p], p), "clocks": res[p]["clocks"]} for p in res},
        "precision": prec_report,
        "precision_256_g0": prec256,
        "precision_256_g01": prec256g,
        "cufft_reference": fft_ref,
        "adjoint": adj,
        "batch": batch,
        "snapshots": snaps,
        "ic": ic,
        "roofline": roofline(res[head], head),
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 16 * cells / K,
                "d2h_bytes_per_step": 16 * cells / K,
                "note": f"set_psi from pinned host complex128, {K} steps, get_psi to pinned host, per step = /K"},
        "gpu_launches": 10 * K,
        "clocks": res[head]["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_port(N, psi0, C)
    # the figures the metric names, last on the line (readers that keep its tail see them)
    gates = {}
    if prec_report:
        gates["512_g001_fp32"] = prec_report["fp32"]["density_relL2"]
        gates["512_g001_mixed"] = prec_report["mixed"]["density_relL2"]
    for key, rep in (("256_g0", prec256), ("256_g01", prec256g)):
        if rep:
            gates[key + "_fp32"] = rep["fp32"]["density_relL2"]
            gates[key + "_mixed"] = rep["mixed"]["density_relL2"]
    out["summary"] = {"ms_per_step": {p: round(res[p]["ms"] / K, 4) for p in res},
                      "fp32_over_fp64": round(vals["fp32"] / fp64_value, 4),
                      "density_relL2_after_1000_steps": {k: float("%.3g" % v) for k, v in gates.items()},
                      "gate": gate, "headline_path": head,
                      "adjoint_over_forward": round(adj["adjoint_over_forward"], 3) if adj else None,
                      "e2e_over_value": round(e2e_value / value, 3)}
    rep_.close()
    if rank == 0:
        print(json.dumps(out))


def run_batch(args, prec, device, adjoint_steps=0):
    """96 realisations of uneven sizes (32 at 32^3, 32 at 48^3, 24 at 64^3, 8 at
    96^3), each with its own seed and mfdm ~ U[1e-24, 5e-24] eV, g = 0, K steps
    with per-box step scales under which 500 kinetic-limited steps would reach
    a = 0.5 (potential-limited steps advance less): one tuned graph launch per
    K steps against the same runs one at a time (each run's K steps, then a
    synchronize)."""
    import numpy as np

    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    K = args.batch_steps
    sizes = [32] * 32 + [48] * 32 + [64] * 24 + [96] * 8
    rng = np.random.default_rng(4000)
    masses = rng.uniform(1e-24, 5e-24, len(sizes))
    dts = [dt_scale_for(n, 500, mfdm=float(m)) for n, m in zip(sizes, masses)]
    psis = [zeldovich_psi(n, xmax=XMAX, seed=4000 + i, a=A0, mfdm=float(m))
            for i, (n, m) in enumerate(zip(sizes, masses))]
    sims = [ifdm.Simulation(float(m), 0.0, XMAX, n, precision=prec, device=device) for n, m in zip(sizes, masses)]

    def reset():
        for sim, psi in zip(sims, psis):
            sim.set_psi(psi, A0)
        for sim in sims:
            sim.synchronize()

    reset()
    b = ifdm.Batch(sims)
    tuning = b.tune(5, dts)
    b.step(K, dts)  # captures and instantiates the graph for K steps
    b.synchronize()
    reset()
    t0 = time.perf_counter()
    b.step(K, dts)
    b.synchronize()
    t_batch = time.perf_counter() - t0
    out_batch = [sim.get_psi() for sim in sims]
    info = b.info()
    # the same schedule with the default radix plans: the arithmetic of the one-box runs
    b.set_tuning(mode=tuning["mode"], blocks_per_sm=tuning["blocks_per_sm"], group=tuning["group"], plan=(0,) * 6)
    reset()
    b.step(K, dts)
    b.synchronize()
    out_default = [sim.get_psi() for sim in sims]
    b.close()
    reset()
    t0 = time.perf_counter()
    for sim, dt in zip(sims, dts):
        sim.step(K, dt)
        sim.synchronize()
    t_single = time.perf_counter() - t0
    single = [sim.get_psi() for sim in sims]

    def max_rel(xs, ys):
        return max(float(np.linalg.norm(x - y) / np.linalg.norm(y)) for x, y in zip(xs, ys))

    def max_rel_rho(xs, ys):
        return max(float(np.linalg.norm(np.abs(x) ** 2 - np.abs(y) ** 2) / np.linalg.norm(np.abs(y) ** 2))
                   for x, y in zip(xs, ys))

    a_end = min(sim.state()["a"] for sim in sims)
    adj = None
    if adjoint_steps > 0:
        # batched adjoint (record + backward sweep of every box side by side)
        # against the boxes' own record + adjoint calls one after another;
        # host cotangents in and gradients out in both
        grng = np.random.default_rng(5000)
        gfin = [grng.standard_normal((n,) * 3) + 1j * grng.standard_normal((n,) * 3) for n in sizes]
        g0b = [np.empty((n,) * 3, dtype=np.complex128) for n in sizes]
        g0s = [np.empty((n,) * 3, dtype=np.complex128) for n in sizes]
        ba = ifdm.Batch(sims)
        # untimed warm-up of both legs: the first record allocates each box's
        # checkpoint and segment buffers
        reset()
        ba.record_steps(adjoint_steps, dts, 20)
        ba.adjoint(gfin, g0b)
        reset()
        t0 = time.perf_counter()
        ba.record_steps(adjoint_steps, dts, 20)
        ba.adjoint(gfin, g0b)
        t_badj = time.perf_counter() - t0
        ba.close()
        reset()
        t0 = time.perf_counter()
        for sim, dt, gf, g in zip(sims, dts, gfin, g0s):
            sim.record_steps(adjoint_steps, dt, 20)
            sim.adjoint(gf, g)
        t_sadj = time.perf_counter() - t0
        adj = {"steps": adjoint_steps, "checkpoint_every": 20, "batch_s": t_badj, "one_at_a_time_s": t_sadj,
               "speedup": t_sadj / t_badj, "identical": all(np.array_equal(x, y) for x, y in zip(g0b, g0s))}
    for sim in sims:
        sim.close()
    cells = float(sum(n ** 3 for n in sizes))
    return {"path": prec, "boxes": len(sizes), "sizes": {"32": 32, "48": 32, "64": 24, "96": 8}, "steps": K,
            "value": cells * K / t_batch, "unit": "cell-steps/s", "batch_s": t_batch, "one_at_a_time_s": t_single,
            "speedup": t_single / t_batch, "one_at_a_time_value": cells * K / t_single,
            "psi_rel_l2_vs_one_at_a_time": {"default_plans": max_rel(out_default, single),
                                            "tuned_plans": max_rel(out_batch, single)},
            "density_rel_l2_vs_one_at_a_time": {"default_plans": max_rel_rho(out_default, single),
                                                "tuned_plans": max_rel_rho(out_batch, single)},
            "min_a_end": a_end, "tuning": tuning, "adjoint": adj,
            "items_per_step": info["items_per_step"], "persistent_ctas": info["grid"],
            "note": "wall clock around one graph replay (state reset between runs, graph captured beforehand)"}


def run_reference(args):
    """The reference's own code on the host cores (rank 0 only)."""
    import numpy as np

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ifdm_code_b200.synthetic_ic import zeldovich_psi
    from oracle import ref_binary

    N = args.res
    binary = ref_binary()
    if binary is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/BECMPI_ref was not built"}))
        return
    K = max(1, min(args.steps, args.ref_max_steps))
    W = 1
    with tempfile.TemporaryDirectory() as d:
        psi0 = zeldovich_psi(N, xmax=XMAX, seed=0, a=A0, mfdm=MFDM)
        G = g_for_phase(N, psi0, dt_scale_for(N), args.g_phase)  # the same self-interaction as the GPU arm
        xm = XMAX / 0.677
        x = xm / N - xm + np.arange(N) * (2 * xm / N)
        with open(os.path.join(d, "output1.dat"), "wb") as f:
            np.array([MFDM, 0.0, A0], dtype=np.float64).tofile(f)
            x.astype(np.float64).tofile(f)
            psi0.tofile(f)
        del psi0
        tf = os.path.join(d, "steps.txt")
        env = dict(os.environ, IFDM_SHIM_TIMING=tf)
        # rerun from output1.dat; t_write larger than the run so only the last
        # step writes (that step is not timed)
        cmd = [binary, str(MFDM), repr(G), str(XMAX), str(N), "1000000", str(1 + W + K + 1), "1", d + "/", d + "/", "1"]
        subprocess.run(cmd, env=env, capture_output=True, text=True, check=True)
        ts = [float(v) for v in open(tf).read().split()]
    starts = ts[0::2]
    dts = [b - a for a, b in zip(starts[:-1], starts[1:])][W:W + K]
    sec = statistics.mean(dts)
    value = float(N) ** 3 / sec
    cores = os.cpu_count()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": 0,
        "steps": len(dts), "warmup": W, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{N}^3 leap-frog step (reference loop, rerun from a synthetic snapshot), "
                               f"g={G:.4e} eV cm^3 ({args.g_phase} rad/step at the densest cell)",
                   "res": N, "g_eV_cm3": G,
                   "steps_cap": f"at most --ref-max-steps={args.ref_max_steps} timed steps: one reference step "
                                f"takes ~13 s at 512^3 on this host, so the arm stays within a few minutes",
                   "reference_build": "the reference's MPI-FFTW build is unavailable on this box (no MPI, FFTW3 "
                                      "or GSL); its own sources run against single-rank shims"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": "reference",
                         "sample": f"{len(dts)} timed steps after {W} warm-up at {N}^3; FFTs on {cores} OpenMP "
                                   "threads (shim), pointwise loops on 1 thread as one MPI rank runs them"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_stability(args):
    """FP64 record of the split-step scheme's stability at N^3 under the
    self-interaction strengths 0.1, 0.03 and 0.01 rad per step at the densest
    cell (the benchmark's fixed-step schedule): max|psi|^2 relative to its
    initial value, a and the limiting criterion every 10 steps."""
    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    N = args.res
    C = dt_scale_for(N)
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=0, a=A0, mfdm=MFDM)
    out = {"res": N, "dt_scale": C, "steps": args.precision_steps, "every": 10, "runs": {}}
    for phase in (0.1, 0.03, 0.01):
        G = g_for_phase(N, psi0, C, phase)
        trace = []
        with ifdm.Simulation(MFDM, G, XMAX, N) as sim:
            sim.set_psi(psi0, A0)
            sim.step(1, C)
            r0 = sim.state()["max_rho"]
            for n in range(1, args.precision_steps, 10):
                st = sim.state()
                trace.append([int(st["steps"]), round(st["max_rho"] / r0, 4), round(st["a"], 6), int(st["criterion"])])
                sim.step(min(10, args.precision_steps - n), C)
            st = sim.state()
            trace.append([int(st["steps"]), round(st["max_rho"] / r0, 4), round(st["a"], 6), int(st["criterion"])])
        out["runs"][str(phase)] = {"g_eV_cm3": G, "trace": trace}
    print(json.dumps(out))


def run_profile(args):
    """Short fixed run of one precision for ncu captures: W + K steps, no timing."""
    import ifdm_code_b200 as ifdm
    from ifdm_code_b200.synthetic_ic import zeldovich_psi

    N = args.res
    C = dt_scale_for(N)
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=0, a=A0, mfdm=MFDM)
    with ifdm.Simulation(MFDM, 0.0, XMAX, N, precision=args.precision) as sim:
        sim.set_psi(psi0, A0)
        sim.step(args.warmup + args.steps, C)
        sim.synchronize()
        print(json.dumps({"profile": True, "res": N, "precision": args.precision, "steps": args.warmup + args.steps,
                          "a": sim.state()["a"]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--res", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true", help="plain W+K steps of --precision (for ncu)")
    ap.add_argument("--profile-ic", action="store_true", help="only the IC section at --ic-res (for ncu)")
    ap.add_argument("--calibrate-g", action="store_true", help="print the g of the self-interaction config")
    ap.add_argument("--stability", action="store_true",
                    help="FP64 max|psi|^2 trace at --res under 0.1/0.03/0.01 rad per step (no timing)")
    ap.add_argument("--precision", choices=["fp32", "fp64", "mixed"], default="mixed")
    ap.add_argument("--adjoint-steps", type=int, default=40, help="steps of the adjoint timing (0 skips it)")
    ap.add_argument("--g-phase", type=float, default=0.01,
                    help="self-interaction: radians per step at the densest cell in the first (largest) turn, "
                         "0: g = 0.  The configuration asks ~0.1; at 512^3 the split-step scheme (the "
                         "reference's and this one) turns unstable above ~0.02 (max|psi|^2 x100 within 150 "
                         "steps at 0.1), so the benchmark uses 0.01")
    ap.add_argument("--batch-steps", type=int, default=500, help="steps of the 96-box batch timing (0 skips it)")
    ap.add_argument("--ic-res", type=int, default=512,
                    help="particles per side of the IC pre-processing timing (0 skips it)")
    ap.add_argument("--snapshot-steps", type=int, default=4,
                    help="snapshots per schedule of the blocking vs streamed timing (0 skips it)")
    ap.add_argument("--precision-steps", type=int, default=1000,
                    help="steps of the precision gate (density error vs FP64); 0 skips it")
    ap.add_argument("--ref-max-steps", type=int, default=6,
                    help="bound on timed reference steps (each is ~tens of seconds at 512^3)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.profile:
        run_profile(args)
    elif args.profile_ic:
        import ifdm_code_b200 as ifdm

        print(json.dumps(ic_section(ifdm, args.ic_res, 0, 0)))
    elif args.stability:
        run_stability(args)
    elif args.calibrate_g:
        calibrate_g(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
