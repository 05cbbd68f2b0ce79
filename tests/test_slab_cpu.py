"""Slab decomposition of one box over ranks (the reference's x-slabs,
src/struct3D.h:3-15), host logic on CPU with two and four gloo ranks.

The local passes are numpy stand-ins for the CUDA kernels of ifdm_fft_slab
(one axis of the slab at a time; the x axis on the transposed y-slab, with the
Poisson multiplier and the rank's global y offset); the layout, the
all-to-all transposes and the order of the passes are the module's own.  The
distributed forward transform, inverse transform and Poisson solve must equal
numpy's transforms of the whole box.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

N = 16


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _kappa(n):
    k = np.arange(n)
    return np.where(k < n // 2, k, k - n)


def numpy_axis_op(t, axis, sign, n, planes, poisson=False, y0=0):
    """What ifdm_fft_slab computes, in numpy, written back into the tensor."""
    a = t.numpy()
    f = np.fft.fft if sign < 0 else (lambda x, axis: np.fft.ifft(x, axis=axis) * x.shape[axis])
    if poisson:
        b = np.fft.fft(a, axis=0)
        kx = _kappa(n)[:, None, None]
        ky = _kappa(n)[y0:y0 + planes][None, :, None]
        kz = _kappa(n)[None, None, :]
        k2 = (kx * kx + ky * ky + kz * kz).astype(np.float64)
        m = np.where(k2 == 0, 0.0, -1.0 / np.where(k2 == 0, 1.0, k2) / n**3)
        a[...] = np.fft.ifft(b * m, axis=0) * n
    else:
        a[...] = f(a, axis=axis)  # tensor dim = library axis (x on the y-slab is dim 0)
    return t


def _full(seed=5):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N))


def _poisson_numpy(rho):
    k = _kappa(N)
    k2 = (k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2).astype(np.float64)
    k2[0, 0, 0] = 1.0
    r = -np.fft.fftn(rho) / k2
    r[0, 0, 0] = 0.0
    return np.fft.ifftn(r)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist

    from ifdm_code_b200.slab import SlabFFT, SlabLayout, x_to_y, y_to_x

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    lay = SlabLayout(N, world, rank)
    full = _full()
    fft = SlabFFT(lay, axis_op=numpy_axis_op)
    loc = torch.from_numpy(lay.local(full).copy())
    # the transposes alone: y-slab of rank r = planes [x0, x0+n0) of y for every x
    y = x_to_y(loc.clone(), lay)
    ok_t = np.array_equal(y.numpy(), full[:, lay.x0:lay.x0 + lay.n0, :])
    ok_back = np.array_equal(y_to_x(y, lay).numpy(), lay.local(full))
    fwd = fft.transform(loc.clone(), -1).numpy()
    inv = fft.transform(torch.from_numpy(fwd.copy()), +1).numpy() / N**3
    rho = np.abs(full) ** 2
    phi = fft.poisson(torch.from_numpy(lay.local(rho).astype(np.complex128).copy())).numpy()
    ref_fwd = lay.local(np.fft.fftn(full))
    ref_phi = lay.local(_poisson_numpy(rho))
    out[rank] = (ok_t, ok_back, float(np.abs(fwd - ref_fwd).max() / np.abs(ref_fwd).max()),
                 float(np.abs(inv - lay.local(full)).max()), float(np.abs(phi - ref_phi).max() / np.abs(ref_phi).max()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_slab_transforms_over_gloo_ranks(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ok_t, ok_back, e_fwd, e_inv, e_phi = out[r]
        assert ok_t and ok_back, r
        assert e_fwd <= 1e-13 and e_inv <= 1e-13 and e_phi <= 1e-13, (r, e_fwd, e_inv, e_phi)


def test_layout_matches_the_reference_slabs():
    from ifdm_code_b200.slab import SlabLayout

    # local_n0 = N / P, local_0_start = rank * local_n0 (src/struct3D.h:3-15)
    lay = SlabLayout(512, 8, 3)
    assert (lay.n0, lay.x0) == (64, 192)
    with pytest.raises(ValueError):
        SlabLayout(512, 3, 0)
    with pytest.raises(ValueError):
        SlabLayout(512, 4, 4)


def test_single_rank_needs_no_exchange():
    import torch

    from ifdm_code_b200.slab import SlabFFT, SlabLayout

    full = _full(7)
    lay = SlabLayout(N, 1, 0)
    got = SlabFFT(lay, axis_op=numpy_axis_op).transform(torch.from_numpy(full.copy()), -1).numpy()
    assert np.abs(got - np.fft.fftn(full)).max() / np.abs(got).max() <= 1e-13
