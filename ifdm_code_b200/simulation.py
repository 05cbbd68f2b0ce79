"""Python mirror of the reference's run interface over the C ABI.

``Simulation`` takes the reference's 10 run-time parameters
(``src/CosmoBEC_MPI.cpp:329-339``) and exposes its phases: IC generation
(``Gadget_IC_Generator``), rerun (``read_rerun``), the stepping loop with its
snapshot state machine (``Simulation``), snapshot writes (``writeall``), plus
fixed-step stepping and state access for tests and benchmarks.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import BatchTuning, Energies, IfdmError, Params, State


def _check(lib, h, rc: int) -> int:
    if rc < 0:
        msg = lib.ifdm_last_error(h)
        raise IfdmError(rc, msg.decode() if msg else "")
    return rc


class Simulation:
    """One box on one GPU.

    precision: "fp64" (the drop-in path), "fp32" (FP32 arithmetic) or "mixed"
               (FP32 storage, FP64 arithmetic, stochastic FP32 rounding).
    ic_mode:   "ref1" reproduces the reference run on one MPI rank, "exact"
               deposits every IC particle once.
    """

    def __init__(self, mfdm: float, g: float, xmax: float, res: int, t_write: int = 1, t_stop: int = 1,
                 ti: int = 0, opath: str = "", icpath: str = "", rerun: int = 0, precision: str = "fp64",
                 stan: bool = False, ic_mode: str = "ref1", device: int = 0, verbose: bool = False):
        self.lib = _lib.load_library()
        self._strs = [opath.encode(), icpath.encode()]
        p = Params()
        self.lib.ifdm_params_default(C.byref(p))
        p.mfdm, p.g, p.xmax, p.res = mfdm, g, xmax, res
        p.t_write, p.t_stop, p.ti = t_write, t_stop, ti
        p.opath, p.icpath, p.rerun = self._strs[0], self._strs[1], rerun
        p.precision = {"fp64": _lib.FP64, "fp32": _lib.FP32, "mixed": _lib.MIXED}[precision]
        p.stan = int(stan)
        p.ic_mode = {"ref1": _lib.IC_REF1, "exact": _lib.IC_EXACT}[ic_mode]
        p.device = device
        p.verbose = int(verbose)
        self.N = res
        self.precision = precision
        h = C.c_void_p()
        rc = self.lib.ifdm_create(C.byref(p), C.byref(h))
        self.h = h.value
        if rc < 0:
            msg = self.lib.ifdm_last_error(self.h)
            self.close()
            raise IfdmError(rc, msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ifdm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, rc: int) -> int:
        return _check(self.lib, self.h, rc)

    # ---------------------------------------------------------------- state --
    def load_ic(self) -> None:
        self._c(self.lib.ifdm_load_ic(self.h))

    def load_snapshot(self, t: int) -> None:
        self._c(self.lib.ifdm_load_snapshot(self.h, t))

    def set_psi(self, psi, a: float, rhoc: float = 0.0) -> None:
        """psi: complex128 array (host numpy) or CUDA tensor of N^3 elements."""
        if hasattr(psi, "data_ptr"):
            ptr = psi.data_ptr()
            self._c(self.lib.ifdm_set_psi(self.h, C.c_void_p(ptr), a, rhoc))
        else:
            buf = np.ascontiguousarray(psi, dtype=np.complex128)
            self._c(self.lib.ifdm_set_psi(self.h, buf.ctypes.data_as(C.c_void_p), a, rhoc))

    def get_psi(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.N,) * 3, dtype=np.complex128)
        self._c(self.lib.ifdm_get_psi(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def get_psi_into(self, tensor) -> None:
        """psi after the latest step into a contiguous complex128 CUDA tensor."""
        self._c(self.lib.ifdm_get_psi(self.h, C.c_void_p(tensor.data_ptr())))

    def record_steps(self, nsteps: int, dt_scale: float = 1.0, checkpoint_every: int = 20) -> None:
        """nsteps fixed-mode steps that keep what ``adjoint`` needs."""
        self._c(self.lib.ifdm_record_steps(self.h, nsteps, dt_scale, checkpoint_every))

    def adjoint(self, g_final, g0) -> None:
        """dL/dpsi_final -> dL/dpsi_0 through the recorded steps (complex128
        numpy arrays or CUDA tensors, dL/dRe + i dL/dIm)."""
        def ptr(a):
            return C.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else a.ctypes.data_as(C.c_void_p)
        self._c(self.lib.ifdm_adjoint(self.h, ptr(g_final), ptr(g0)))

    def get_phi(self) -> np.ndarray:
        out = np.empty((self.N,) * 3, dtype=np.float64)
        self._c(self.lib.ifdm_get_phi(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def power_spectrum(self, nbins: int = 24, edges=None) -> dict:
        """P(k) of the density contrast of the current state, on the device.
        edges: nbins+1 increasing |kappa| bin edges (integer wave-vector
        units); None: log-spaced from 1 to N/2.  Returns k [1/Mpc], pk
        [Mpc^3], modes per bin and <|psi|^2>."""
        k = np.zeros(nbins)
        pk = np.zeros(nbins)
        modes = np.zeros(nbins, dtype=np.int64)
        mean = C.c_double()
        e = None
        if edges is not None:
            e = np.ascontiguousarray(edges, dtype=np.float64)
            if e.shape != (nbins + 1,):
                raise ValueError("edges needs nbins + 1 values")
        self._c(self.lib.ifdm_power_spectrum(self.h, nbins, None if e is None else e.ctypes.data_as(C.c_void_p),
                                             k.ctypes.data_as(C.c_void_p), pk.ctypes.data_as(C.c_void_p),
                                             modes.ctypes.data_as(C.c_void_p), C.byref(mean)))
        return {"k": k, "pk": pk, "modes": modes, "mean_rho": mean.value}

    def energies(self) -> dict:
        """Grid means of the current state, on the device: <|psi|^2>,
        <|grad psi|^2> (1/Mpc^2 x psi units), <phi |psi|^2> and <|psi|^4>."""
        e = Energies()
        self._c(self.lib.ifdm_get_energies(self.h, C.byref(e)))
        return {k: getattr(e, k) for k, _ in Energies._fields_}

    def state(self) -> dict:
        s = State()
        self._c(self.lib.ifdm_get_state(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in State._fields_}

    # ------------------------------------------------------------- stepping --
    def run(self) -> None:
        self._c(self.lib.ifdm_run(self.h))

    def step(self, nsteps: int, dt_scale: float = 1.0) -> None:
        self._c(self.lib.ifdm_step(self.h, nsteps, dt_scale))

    def write_snapshot(self, t: int) -> None:
        """<opath>output<t>.dat of the current state, complete on return."""
        self._c(self.lib.ifdm_write_snapshot(self.h, t))

    def write_snapshot_async(self, t: int) -> None:
        """Queue <opath>output<t>.dat; it is written while later steps run."""
        self._c(self.lib.ifdm_write_snapshot_async(self.h, t))

    def flush_snapshots(self) -> None:
        """Wait until every queued snapshot file is written."""
        self._c(self.lib.ifdm_flush_snapshots(self.h))

    def set_snapshot_streaming(self, on: bool) -> None:
        """False: gather and write each snapshot inside the call (the
        reference's blocking writeall)."""
        self._c(self.lib.ifdm_set_snapshot_streaming(self.h, 1 if on else 0))

    @property
    def snapshots_written(self) -> int:
        return int(self.lib.ifdm_snapshots_written(self.h))

    def synchronize(self) -> None:
        self._c(self.lib.ifdm_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.lib.ifdm_stream(self.h) or 0

    def profile_passes(self, nsteps: int, dt_scale: float = 1.0) -> dict:
        ms = (C.c_double * 16)()
        names = (C.c_char_p * 16)()
        n = self._c(self.lib.ifdm_profile_passes(self.h, nsteps, dt_scale, ms, names, 16))
        return {names[i].decode(): ms[i] for i in range(n)}

    def pass_bytes(self) -> list[float]:
        b = (C.c_double * 16)()
        n = self._c(self.lib.ifdm_pass_bytes(self.h, b, 16))
        return [b[i] for i in range(n)]


def fft3d_(tensor, sign: int, compute: str | None = None) -> None:
    """In-place unnormalised 3-D FFT of a contiguous cubic CUDA complex tensor
    (complex128 or complex64) on torch's current stream; compute="fp64" runs a
    complex64 tensor through FP64 arithmetic."""
    import torch

    lib = _lib.load_library()
    if not tensor.is_cuda or not tensor.is_contiguous() or tensor.dim() != 3:
        raise ValueError("need a contiguous 3-D CUDA tensor")
    n = tensor.shape[0]
    prec = {torch.complex128: _lib.FP64, torch.complex64: _lib.FP32}[tensor.dtype]
    if compute == "fp64" and tensor.dtype == torch.complex64:
        prec = _lib.MIXED
    stream = torch.cuda.current_stream(tensor.device).cuda_stream
    rc = lib.ifdm_fft3d(C.c_void_p(tensor.data_ptr()), n, prec, sign, C.c_void_p(stream))
    if rc < 0:
        raise IfdmError(rc, "ifdm_fft3d failed")


def supported_res(res: int, precision: str = "fp64") -> bool:
    return bool(_lib.load_library().ifdm_supported_res(res, {"fp64": 0, "fp32": 1, "mixed": 2}[precision]))


class Batch:
    """Several Simulations (res 16..128, one device, one precision) advanced
    together: one replay of a captured CUDA graph per ``step`` call, in which
    the boxes of each grid size share one persistent kernel (or one launch per
    phase, whichever ``tune`` found faster).  Each box keeps its own state and
    is read through its Simulation as usual."""

    def __init__(self, sims: list[Simulation]):
        self.lib = _lib.load_library()
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s.h for s in self.sims])
        h = C.c_void_p()
        rc = self.lib.ifdm_batch_create(arr, len(self.sims), C.byref(h))
        self.h = h.value
        if rc < 0:
            msg = self.lib.ifdm_batch_last_error(self.h) if self.h else b""
            self.close()
            raise IfdmError(rc, msg.decode() if msg else "")

    def _c(self, rc: int) -> int:
        if rc < 0:
            msg = self.lib.ifdm_batch_last_error(self.h)
            raise IfdmError(rc, msg.decode() if msg else "")
        return rc

    def _dts(self, dt_scale):
        if np.isscalar(dt_scale):
            dt_scale = [float(dt_scale)] * len(self.sims)
        if len(dt_scale) != len(self.sims):
            raise ValueError("one dt_scale per box")
        return (C.c_double * len(self.sims))(*[float(x) for x in dt_scale])

    def step(self, nsteps: int, dt_scale=1.0) -> None:
        """nsteps fixed-mode steps of every box (asynchronous)."""
        self._c(self.lib.ifdm_batch_step(self.h, nsteps, self._dts(dt_scale)))

    def tune(self, trial_steps: int, dt_scale=1.0) -> dict:
        t = BatchTuning()
        self._c(self.lib.ifdm_batch_tune(self.h, trial_steps, self._dts(dt_scale), C.byref(t)))
        return self._tuning_dict(t)

    def get_tuning(self) -> dict:
        t = BatchTuning()
        self._c(self.lib.ifdm_batch_get_tuning(self.h, C.byref(t)))
        return self._tuning_dict(t)

    def set_tuning(self, mode: int = 0, blocks_per_sm: int = 2, group: int = 0, plan=(0,) * 6) -> None:
        t = BatchTuning(mode, blocks_per_sm, group, (C.c_int * 6)(*plan), 0.0)
        self._c(self.lib.ifdm_batch_set_tuning(self.h, C.byref(t)))

    @staticmethod
    def _tuning_dict(t) -> dict:
        return {"mode": t.mode, "blocks_per_sm": t.blocks_per_sm, "group": t.group, "plan": list(t.plan),
                "ms_per_step": t.ms_per_step}

    def record_steps(self, nsteps: int, dt_scale=1.0, checkpoint_every: int = 20) -> None:
        """Every box records nsteps fixed-mode steps for its adjoint, the boxes
        side by side (each on its own stream)."""
        self._c(self.lib.ifdm_batch_record_steps(self.h, nsteps, self._dts(dt_scale), checkpoint_every))

    def adjoint(self, g_finals, g0s) -> None:
        """The adjoint of every box's recorded steps, side by side; g_finals /
        g0s: one complex128 array (numpy or CUDA tensor) per box."""
        if len(g_finals) != len(self.sims) or len(g0s) != len(self.sims):
            raise ValueError("one g_final and one g0 per box")

        def ptr(a):
            return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data

        gin = (C.c_void_p * len(self.sims))(*[ptr(a) for a in g_finals])
        gout = (C.c_void_p * len(self.sims))(*[ptr(a) for a in g0s])
        self._c(self.lib.ifdm_batch_adjoint(self.h, gin, gout))

    def info(self) -> dict:
        items, grid = C.c_longlong(), C.c_int()
        self._c(self.lib.ifdm_batch_info(self.h, C.byref(items), C.byref(grid)))
        return {"items_per_step": items.value, "grid": grid.value}

    def synchronize(self) -> None:
        self._c(self.lib.ifdm_batch_synchronize(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ifdm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

