"""Slab-local kernels of the slab decomposition on a B200 (needs a B200).

ifdm_fft_slab on the slabs a 4-rank split of a 64^3 box gives each rank (the
z and y axes on the x-slab, the x axis and the fused Poisson x pass on the
transposed y-slab with the rank's global y offset) against numpy, and the
distributed transform and Poisson solve of ifdm_code_b200.slab on one rank
against the one-box 3-D FFT.  The exchange between ranks is covered by the
gloo tests (tests/test_slab_cpu.py): the runs here have one GPU.
"""

import numpy as np
import pytest

import ifdm_code_b200 as ifdm
from tests.test_slab_cpu import numpy_axis_op

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-13, "fp32": 3e-6}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_slab_axis_kernels_match_numpy(prec):
    import torch

    from ifdm_code_b200.slab import SlabLayout, library_axis_op

    n, world = 64, 4
    dt = torch.complex128 if prec == "fp64" else torch.complex64
    rng = np.random.default_rng(64)
    full = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    op = library_axis_op(prec)
    for rank in range(world):
        lay = SlabLayout(n, world, rank)
        cases = [(lay.local(full), 2, -1, False), (lay.local(full), 1, +1, False),
                 (full[:, lay.x0:lay.x0 + lay.n0, :], 0, -1, False), (full[:, lay.x0:lay.x0 + lay.n0, :], 0, 0, True)]
        for data, axis, sign, poisson in cases:
            t = torch.from_numpy(np.ascontiguousarray(data)).to(device="cuda", dtype=dt)
            op(t, axis, sign if sign else -1, n, lay.n0, poisson, lay.x0)
            torch.cuda.synchronize()
            ref = numpy_axis_op(torch.from_numpy(np.ascontiguousarray(data).copy()), axis, sign if sign else -1, n,
                                lay.n0, poisson, lay.x0).numpy()
            err = np.linalg.norm(t.cpu().numpy() - ref) / np.linalg.norm(ref)
            assert err <= TOL[prec], (rank, axis, poisson, err)


def test_slab_fft_one_rank_equals_the_box_fft():
    import torch

    from ifdm_code_b200.slab import SlabFFT, SlabLayout

    n = 128
    rng = np.random.default_rng(128)
    full = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    fft = SlabFFT(SlabLayout(n, 1, 0))
    a = torch.from_numpy(full).cuda()
    b = a.clone()
    fft.transform(a, -1)
    ifdm.fft3d_(b, -1)
    torch.cuda.synchronize()
    assert torch.equal(a, b)  # the same plain kernels in the same order
    rho = np.abs(rng.standard_normal((n, n, n)))
    phi = fft.poisson(torch.from_numpy(rho.astype(np.complex128)).cuda())
    torch.cuda.synchronize()
    ref = _poisson_numpy_n(rho)
    assert np.linalg.norm(phi.cpu().numpy() - ref) / np.linalg.norm(ref) <= 1e-13


def _poisson_numpy_n(rho):
    n = rho.shape[0]
    k = np.arange(n)
    k = np.where(k < n // 2, k, k - n)
    k2 = (k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2).astype(np.float64)
    k2[0, 0, 0] = 1.0
    r = -np.fft.fftn(rho) / k2
    r[0, 0, 0] = 0.0
    return np.fft.ifftn(r)


def test_slab_bad_arguments():
    import ctypes as C

    import torch

    lib = ifdm.load_library()
    t = torch.zeros((16, 64, 64), dtype=torch.complex128, device="cuda")
    p = C.c_void_p(t.data_ptr())
    assert lib.ifdm_fft_slab(p, 64, 16, 3, 0, -1, 0, 0, None) == -1  # axis
    assert lib.ifdm_fft_slab(p, 64, 16, 1, 0, -1, 1, 0, None) == -1  # Poisson op only on x
    assert lib.ifdm_fft_slab(p, 64, 16, 0, 0, -1, 1, 56, None) == -1  # y planes beyond the box
    assert lib.ifdm_fft_slab(p, 16, 4, 2, 0, -1, 0, 0, None) == -1  # 64 lines: not a multiple of the 16^3 tile
    assert lib.ifdm_fft_slab(p, 60, 15, 2, 0, -1, 0, 0, None) == -5  # no plan
