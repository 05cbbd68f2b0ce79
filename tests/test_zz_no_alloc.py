"""ifdm_poisson_static: the potential without any device allocation (needs a B200).

Some callers cannot allocate device memory themselves -- their device memory
belongs to another allocator (a framework's caching pool), or they run in a
time-critical loop where cudaMalloc/cudaFree, which may synchronise the whole
device, are not acceptable.  ifdm_poisson_static serves them from a static
scratch array inside the library.  Its result must equal what the allocating
path (a Simulation context: set_psi then get_phi) returns for the same wave
function, on consecutive calls that reuse the shared scratch.

This file is collected last so that a failure here cannot hide other results.
"""

import ctypes as C

import numpy as np
import pytest

import ifdm_code_b200 as ifdm
from ifdm_code_b200 import _lib
from ifdm_code_b200.synthetic_ic import zeldovich_psi
from tests.snapshot_util import rel_l2

pytestmark = pytest.mark.gpu

MFDM, XMAX, A0 = 2.5e-24, 5.0, 1.0 / 51.0
PHI_TOL = 1e-12  # the tolerance test_phi_matches_oracle holds phi to


def _phi_allocating(psi: np.ndarray) -> np.ndarray:
    with ifdm.Simulation(MFDM, 0.0, XMAX, psi.shape[0]) as s:
        s.set_psi(psi, A0)
        return s.get_phi()


def _call(psi_d, phi_d, n):
    import torch

    lib = ifdm.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.ifdm_poisson_static(C.c_void_p(psi_d.data_ptr()), C.c_void_p(phi_d.data_ptr()), n, MFDM, XMAX,
                                 C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc


def _phi_static(psi: np.ndarray):
    import torch

    n = psi.shape[0]
    psi_d = torch.from_numpy(psi).cuda()
    phi_d = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
    rc = _call(psi_d, phi_d, n)
    return rc, phi_d.cpu().numpy()


def test_static_poisson_matches_allocating_path_on_consecutive_calls():
    # calls in a row share (and overwrite) the static scratch: two at the
    # largest size, then every other size, each with its own kernels
    for n, seed in ((64, 1), (64, 2), (48, 3), (32, 4), (16, 5), (32, 6)):
        psi = zeldovich_psi(n, seed=seed)
        rc, phi = _phi_static(psi)
        assert rc == _lib.IFDM_OK
        ref = _phi_allocating(psi)
        assert rel_l2(phi, ref) <= PHI_TOL, (n, seed)


def test_static_poisson_allocates_no_device_memory():
    """After a first call (the per-device set-up), further calls leave the
    device's free memory and torch's allocator untouched."""
    import torch

    bufs = {}
    for n in (64, 32):
        psi_d = torch.from_numpy(zeldovich_psi(n, seed=7)).cuda()
        phi_d = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
        bufs[n] = (psi_d, phi_d)
        assert _call(psi_d, phi_d, n) == _lib.IFDM_OK  # warm-up: kernels of this size loaded
    free0 = torch.cuda.mem_get_info()[0]
    stats0 = torch.cuda.memory_stats()
    for n in (64, 32, 64):
        assert _call(*bufs[n], n) == _lib.IFDM_OK
    assert torch.cuda.mem_get_info()[0] == free0
    stats1 = torch.cuda.memory_stats()
    for key in ("allocation.all.allocated", "segment.all.allocated"):
        assert stats1.get(key, 0) == stats0.get(key, 0), key


def test_static_poisson_rejects_sizes_beyond_its_scratch():
    import torch

    lib = ifdm.load_library()
    for n in (96, 128):
        psi_d = torch.zeros((n, n, n), dtype=torch.complex128, device="cuda")
        phi_d = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
        rc = lib.ifdm_poisson_static(C.c_void_p(psi_d.data_ptr()), C.c_void_p(phi_d.data_ptr()), n, MFDM, XMAX,
                                     None)
        assert rc == -5  # IFDM_ERR_UNSUPPORTED
    psi_d = torch.zeros((16, 16, 16), dtype=torch.complex128, device="cuda")
    phi_d = torch.empty((16, 16, 16), dtype=torch.float64, device="cuda")
    for n in (0, -16):
        rc = lib.ifdm_poisson_static(C.c_void_p(psi_d.data_ptr()), C.c_void_p(phi_d.data_ptr()), n, MFDM, XMAX,
                                     None)
        assert rc == -1  # IFDM_ERR_ARGS
