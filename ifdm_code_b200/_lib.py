"""ctypes binding of libifdm_b200.so (include/ifdm.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails with an exception when the library is missing; every call that returns
an error status raises IfdmError with the library's message.
"""

from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libifdm_b200.so")
BIN_PATH = os.path.join(PKG, "bin", "BECMPI")

IFDM_OK = 0
ERRORS = {
    -1: "IFDM_ERR_ARGS", -2: "IFDM_ERR_CUDA", -3: "IFDM_ERR_IO", -4: "IFDM_ERR_BOXSIZE",
    -5: "IFDM_ERR_UNSUPPORTED", -6: "IFDM_ERR_STATE", -7: "IFDM_ERR_DEVICE",
}
FP64, FP32, MIXED = 0, 1, 2
IC_REF1, IC_EXACT = 0, 1

# every entry point include/ifdm.h declares
EXPORTS = [
    "ifdm_params_default", "ifdm_params_from_argv", "ifdm_create", "ifdm_destroy", "ifdm_last_error",
    "ifdm_supported_res", "ifdm_load_ic", "ifdm_load_snapshot", "ifdm_set_psi", "ifdm_get_psi", "ifdm_get_phi",
    "ifdm_get_state", "ifdm_power_spectrum", "ifdm_get_energies", "ifdm_run", "ifdm_step", "ifdm_write_snapshot", "ifdm_write_snapshot_async",
    "ifdm_flush_snapshots", "ifdm_set_snapshot_streaming", "ifdm_snapshots_written", "ifdm_synchronize", "ifdm_stream",
    "ifdm_profile_passes", "ifdm_pass_bytes", "ifdm_fft3d", "ifdm_fft_slab", "ifdm_poisson_static", "ifdm_record_steps",
    "ifdm_adjoint", "ifdm_batch_create", "ifdm_batch_step", "ifdm_batch_tune", "ifdm_batch_get_tuning",
    "ifdm_batch_set_tuning", "ifdm_batch_synchronize", "ifdm_batch_record_steps", "ifdm_batch_adjoint", "ifdm_batch_info", "ifdm_batch_last_error",
    "ifdm_batch_destroy",
]


class IfdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("mfdm", C.c_double), ("g", C.c_double), ("xmax", C.c_double), ("res", C.c_int),
        ("t_write", C.c_int), ("t_stop", C.c_int), ("ti", C.c_int), ("opath", C.c_char_p),
        ("icpath", C.c_char_p), ("rerun", C.c_int), ("precision", C.c_int), ("stan", C.c_int),
        ("ic_mode", C.c_int), ("device", C.c_int), ("verbose", C.c_int),
    ]


class Energies(C.Structure):
    _fields_ = [("mean_rho", C.c_double), ("mean_grad2", C.c_double), ("mean_phi_rho", C.c_double),
                ("mean_rho2", C.c_double)]


class State(C.Structure):
    _fields_ = [
        ("a", C.c_double), ("dt_KE", C.c_double), ("dt_PE", C.c_double), ("dt_QI", C.c_double),
        ("max_phi", C.c_double), ("max_rho", C.c_double), ("rhoc", C.c_double), ("steps", C.c_longlong),
        ("criterion", C.c_int), ("device_error", C.c_int),
    ]


class BatchTuning(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("blocks_per_sm", C.c_int), ("group", C.c_int), ("plan", C.c_int * 6),
        ("ms_per_step", C.c_double),
    ]


_lib = None


def load_library() -> C.CDLL:
    """Load libifdm_b200.so (built by ``python -m ifdm_code_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m ifdm_code_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.ifdm_params_default.argtypes = [C.POINTER(Params)]
    lib.ifdm_params_default.restype = None
    lib.ifdm_params_from_argv.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(Params)]
    lib.ifdm_create.argtypes = [C.POINTER(Params), C.POINTER(P)]
    lib.ifdm_destroy.argtypes = [P]
    lib.ifdm_destroy.restype = None
    lib.ifdm_last_error.argtypes = [P]
    lib.ifdm_last_error.restype = C.c_char_p
    lib.ifdm_supported_res.argtypes = [C.c_int, C.c_int]
    lib.ifdm_load_ic.argtypes = [P]
    lib.ifdm_load_snapshot.argtypes = [P, C.c_int]
    lib.ifdm_set_psi.argtypes = [P, C.c_void_p, C.c_double, C.c_double]
    lib.ifdm_get_psi.argtypes = [P, C.c_void_p]
    lib.ifdm_get_phi.argtypes = [P, C.c_void_p]
    lib.ifdm_get_state.argtypes = [P, C.POINTER(State)]
    lib.ifdm_power_spectrum.argtypes = [P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ifdm_get_energies.argtypes = [P, C.POINTER(Energies)]
    lib.ifdm_run.argtypes = [P]
    lib.ifdm_step.argtypes = [P, C.c_int, C.c_double]
    lib.ifdm_write_snapshot.argtypes = [P, C.c_int]
    lib.ifdm_write_snapshot_async.argtypes = [P, C.c_int]
    lib.ifdm_flush_snapshots.argtypes = [P]
    lib.ifdm_set_snapshot_streaming.argtypes = [P, C.c_int]
    lib.ifdm_snapshots_written.argtypes = [P]
    lib.ifdm_snapshots_written.restype = C.c_longlong
    lib.ifdm_synchronize.argtypes = [P]
    lib.ifdm_stream.argtypes = [P]
    lib.ifdm_stream.restype = C.c_void_p
    lib.ifdm_profile_passes.argtypes = [P, C.c_int, C.c_double, D, C.POINTER(C.c_char_p), C.c_int]
    lib.ifdm_pass_bytes.argtypes = [P, D, C.c_int]
    lib.ifdm_fft3d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    lib.ifdm_fft_slab.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_void_p]
    lib.ifdm_poisson_static.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p]
    lib.ifdm_record_steps.argtypes = [P, C.c_int, C.c_double, C.c_int]
    lib.ifdm_adjoint.argtypes = [P, C.c_void_p, C.c_void_p]
    lib.ifdm_batch_create.argtypes = [C.POINTER(P), C.c_int, C.POINTER(P)]
    lib.ifdm_batch_step.argtypes = [P, C.c_int, D]
    lib.ifdm_batch_tune.argtypes = [P, C.c_int, D, C.POINTER(BatchTuning)]
    lib.ifdm_batch_get_tuning.argtypes = [P, C.POINTER(BatchTuning)]
    lib.ifdm_batch_set_tuning.argtypes = [P, C.POINTER(BatchTuning)]
    lib.ifdm_batch_synchronize.argtypes = [P]
    lib.ifdm_batch_record_steps.argtypes = [P, C.c_int, D, C.c_int]
    lib.ifdm_batch_adjoint.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    lib.ifdm_batch_info.argtypes = [P, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
    lib.ifdm_batch_last_error.argtypes = [P]
    lib.ifdm_batch_last_error.restype = C.c_char_p
    lib.ifdm_batch_destroy.argtypes = [P]
    lib.ifdm_batch_destroy.restype = None
    for name in EXPORTS:
        getattr(lib, name)  # raises AttributeError if an export is missing
    _lib = lib
    return lib
