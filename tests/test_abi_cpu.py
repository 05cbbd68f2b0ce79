"""The C-ABI library loads and exports what include/ifdm.h declares; host-only
entry points behave like the reference's main() (CPU only: no compute call)."""

import ctypes as C
import os
import re
import subprocess

import pytest

import ifdm_code_b200 as ifdm
from ifdm_code_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ifdm.h")


def test_library_exports_every_declared_symbol():
    lib = ifdm.load_library()
    declared = set(re.findall(r"\b(ifdm_[a-z0-9_]+)\s*\(", open(HDR).read()))
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert getattr(lib, name) is not None
    out = subprocess.run(["nm", "-D", "--defined-only", ifdm.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ifdm_[a-z0-9_]+)$", out, re.M))
    assert declared <= exported


def _argv(args):
    arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
    return len(args), arr


def test_params_from_argv_matches_reference_parsing():
    """src/CosmoBEC_MPI.cpp:324-340: argc must be 11; atof/atoi conversions."""
    lib = ifdm.load_library()
    p = _lib.Params()
    n, arr = _argv(["BECMPI.o", "2.5e-24", "1e-62", "5.", "128", "100", "1000", "0", "out/", "ic/x", "0"])
    assert lib.ifdm_params_from_argv(n, arr, C.byref(p)) == 0
    assert (p.mfdm, p.g, p.xmax, p.res, p.t_write, p.t_stop, p.ti, p.rerun) == (2.5e-24, 1e-62, 5.0, 128, 100,
                                                                                 1000, 0, 0)
    assert p.opath == b"out/" and p.icpath == b"ic/x"
    n, arr = _argv(["BECMPI.o", "1", "0", "5", "64", "1", "2", "3", "o/", "i/", "1"])
    assert lib.ifdm_params_from_argv(n, arr, C.byref(p)) == 0 and p.rerun == 1 and p.ti == 3


def test_params_from_argv_rejects_wrong_argc():
    lib = ifdm.load_library()
    p = _lib.Params()
    n, arr = _argv(["BECMPI.o", "1", "0", "5"])
    assert lib.ifdm_params_from_argv(n, arr, C.byref(p)) == -1


def test_cli_wrong_argc_prints_reference_message():
    r = subprocess.run([ifdm.BIN_PATH, "1", "2"], capture_output=True, text=True)
    assert r.returncode == 0
    assert r.stdout.strip() == "ERROR: Arguments 3!= 11"


@pytest.mark.parametrize("n,prec,ok", [(16, 0, 1), (48, 0, 1), (96, 0, 1), (512, 0, 1), (20, 0, 0), (1024, 0, 1),
                                       (1024, 1, 1), (1024, 2, 0), (512, 2, 1), (2048, 0, 0), (480, 0, 0)])
def test_supported_sizes(n, prec, ok):
    """Compiled plans: 16 ... 1024 (the reference's production grid); the mixed
    mode stops at 512, where its FP64 exchange tiles still fit shared memory."""
    assert ifdm.load_library().ifdm_supported_res(n, prec) == ok
