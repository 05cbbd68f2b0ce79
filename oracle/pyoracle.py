"""ctypes binding of oracle/liboracle.so (TEST INFRASTRUCTURE ONLY)."""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

IC_REF1 = 0
IC_EXACT = 1


def build(quiet: bool = True) -> None:
    """Build liboracle.so and, when the reference tree exists, oracle/_ref."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def ref_binary(stan: bool = False) -> str | None:
    p = os.path.join(HERE, "_ref", "BECMPI_ref_stan" if stan else "BECMPI_ref")
    return p if os.path.exists(p) else None


class _Args(C.Structure):
    _fields_ = [
        ("mfdm", C.c_double), ("g_in", C.c_double), ("xmax_in", C.c_double),
        ("res", C.c_int), ("t_write", C.c_int), ("t_stop", C.c_int), ("ti", C.c_int),
        ("opath", C.c_char_p), ("icpath", C.c_char_p), ("rerun", C.c_int),
        ("stan", C.c_int), ("ic_mode", C.c_int), ("verbose", C.c_int),
    ]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        lib.orc_create.restype = P
        lib.orc_create.argtypes = [C.POINTER(_Args)]
        lib.orc_destroy.argtypes = [P]
        for fn in ("orc_load_ic", "orc_simulation"):
            getattr(lib, fn).argtypes = [P]
            getattr(lib, fn).restype = C.c_int
        lib.orc_read_rerun.argtypes = [P, C.c_int]
        lib.orc_writeall.argtypes = [P, C.c_int]
        lib.orc_run_fixed.argtypes = [P, C.c_int, C.c_double]
        lib.orc_poisson.argtypes = [P]
        lib.orc_timestep.argtypes = [P, C.c_double]
        lib.orc_split_op.argtypes = [P]
        lib.orc_set_psi.argtypes = [P, D, C.c_double]
        lib.orc_get_psi.argtypes = [P, D]
        lib.orc_get_phi.argtypes = [P, D]
        lib.orc_get_vxg.argtypes = [P, C.POINTER(C.c_float)]
        lib.orc_get_theta.argtypes = [P, D]
        lib.orc_get_a.argtypes = [P]
        lib.orc_get_a.restype = C.c_double
        lib.orc_get_rhoc.argtypes = [P]
        lib.orc_get_rhoc.restype = C.c_double
        lib.orc_get_dts.argtypes = [P, D]
        lib.orc_get_maxes.argtypes = [P, D]
        lib.orc_constants.argtypes = [D]
        lib.orc_num_threads.restype = C.c_int
        _lib = lib
    return _lib


def oracle_constants() -> dict:
    lib = _load()
    out = np.zeros(8)
    lib.orc_constants(out.ctypes.data_as(C.POINTER(C.c_double)))
    keys = ["H_0", "hbar", "bigG", "c", "Omega_m0", "h_0", "rhoc", "cm2Mpc"]
    return dict(zip(keys, out.tolist()))


@dataclass
class OracleArgs:
    mfdm: float = 2.5e-24
    g: float = 0.0
    xmax: float = 5.0
    res: int = 16
    t_write: int = 1
    t_stop: int = 1
    ti: int = 0
    opath: str = ""
    icpath: str = ""
    rerun: int = 0
    stan: int = 0
    ic_mode: int = IC_REF1
    verbose: int = 0


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One oracle simulation (FP64, CPU)."""

    def __init__(self, args: OracleArgs):
        self.lib = _load()
        self.args = args
        self._keep = [args.opath.encode(), args.icpath.encode()]
        ca = _Args(args.mfdm, args.g, args.xmax, args.res, args.t_write, args.t_stop, args.ti,
                   self._keep[0], self._keep[1], args.rerun, args.stan, args.ic_mode, args.verbose)
        self.h = self.lib.orc_create(C.byref(ca))
        self.N = args.res

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def load_ic(self) -> None:
        rc = self.lib.orc_load_ic(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle IC load failed ({rc})")

    def read_rerun(self, t: int) -> None:
        rc = self.lib.orc_read_rerun(self.h, t)
        if rc != 0:
            raise RuntimeError(f"oracle rerun read failed ({rc})")

    def set_psi(self, psi: np.ndarray, a: float) -> None:
        buf = np.ascontiguousarray(psi, dtype=np.complex128).view(np.float64)
        self.lib.orc_set_psi(self.h, _dp(buf), a)

    def psi(self) -> np.ndarray:
        out = np.empty((self.N,) * 3, dtype=np.complex128)
        self.lib.orc_get_psi(self.h, _dp(out.view(np.float64)))
        return out

    def phi(self) -> np.ndarray:
        out = np.empty((self.N,) * 3, dtype=np.float64)
        self.lib.orc_get_phi(self.h, _dp(out))
        return out

    def vxg(self) -> np.ndarray:
        out = np.empty((self.N,) * 3, dtype=np.float32)
        self.lib.orc_get_vxg(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def theta(self) -> np.ndarray:
        out = np.empty((self.N,) * 3, dtype=np.complex128)
        self.lib.orc_get_theta(self.h, _dp(out.view(np.float64)))
        return out

    @property
    def a(self) -> float:
        return self.lib.orc_get_a(self.h)

    @property
    def rhoc(self) -> float:
        return self.lib.orc_get_rhoc(self.h)

    def dts(self) -> np.ndarray:
        out = np.zeros(3)
        self.lib.orc_get_dts(self.h, _dp(out))
        return out

    def maxes(self) -> np.ndarray:
        out = np.zeros(2)
        self.lib.orc_get_maxes(self.h, _dp(out))
        return out

    def poisson(self):
        self.lib.orc_poisson(self.h)

    def timestep(self, dt_scale: float = 1.0):
        self.lib.orc_timestep(self.h, dt_scale)

    def split_op(self):
        self.lib.orc_split_op(self.h)

    def run_fixed(self, nsteps: int, dt_scale: float) -> None:
        self.lib.orc_run_fixed(self.h, nsteps, dt_scale)

    def simulation(self) -> None:
        self.lib.orc_simulation(self.h)

    def writeall(self, t: int) -> None:
        self.lib.orc_writeall(self.h, t)

    @staticmethod
    def num_threads() -> int:
        return _load().orc_num_threads()
