"""One box split into x-slabs over the ranks of a process group.

The reference's only parallel scheme (src/struct3D.h:3-15): rank p of P holds
local_n0 = N/P consecutive x-planes, starting at local_0_start = p * local_n0,
of the [x][y][z] box (z fastest), and its FFTW-MPI plans
(src/CosmoBEC_MPI.cpp:174-177, no TRANSPOSED flags) return a transform in that
same slab layout.  Here every rank keeps its slab on its own GPU and a 3-D
transform is

    z and y on the x-slab [n0][N][N]         ifdm_fft_slab axis 2, 1 (local kernels)
    x-slab -> y-slab                          one all-to-all of the slab
    x on the y-slab [N][n0][N]                ifdm_fft_slab axis 0
    y-slab -> x-slab                          one all-to-all back

so one exchange per direction crosses the interconnect (NCCL over NVLink on
GPUs, gloo on CPU).  The Poisson solve, phi = -F^-1[F[rho]/kappa^2], runs the
forward z and y passes, one transpose, the x pass with the multiplier fused
between its forward and inverse transforms (op 1, global y planes of the
rank), the transpose back and the inverse y and z passes.  Every buffer a
kernel touches is the launching GPU's own: the exchange is a collective on
the slabs, no kernel or tensor map is given another GPU's memory.

The local steps are callables so that the host logic (layout, transposes,
order of the passes) runs unchanged on CPU ranks in the tests, where a numpy
stand-in replaces the CUDA kernels; the default calls the library.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib


@dataclass(frozen=True)
class SlabLayout:
    """x-planes [x0, x0 + n0) of an n^3 box on rank `rank` of `world` (the
    reference's local_n0 / local_0_start).  After the transpose the same rank
    holds the y-planes [x0, x0 + n0) for every x."""

    n: int
    world: int
    rank: int

    def __post_init__(self):
        if self.world < 1 or not (0 <= self.rank < self.world) or self.n % self.world:
            raise ValueError(f"{self.n}^3 does not split into {self.world} equal slabs")

    @property
    def n0(self) -> int:
        return self.n // self.world

    @property
    def x0(self) -> int:
        return self.rank * self.n0

    def local(self, full):
        """This rank's x-slab of a full box (a view)."""
        return full[self.x0:self.x0 + self.n0]


def _all_to_all(recv, send, group):
    import torch.distributed as dist

    dist.all_to_all_single(recv, send, group=group)


def x_to_y(local, lay: SlabLayout, group=None):
    """[n0 x][N y][N z] on every rank -> [N x][n0 y][N z]: block (x of rank p,
    y of rank q) travels from p to q."""
    P, n0, n = lay.world, lay.n0, lay.n
    if P == 1:
        return local
    send = local.reshape(n0, P, n0, n).permute(1, 0, 2, 3).contiguous()  # [dest q][x][y_q][z]
    recv = send.new_empty(send.shape)  # [src p][x_p][y_mine][z]
    _all_to_all(recv, send, group)
    return recv.reshape(n, n0, n)


def y_to_x(ylocal, lay: SlabLayout, group=None):
    """The inverse of x_to_y: [N x][n0 y][N z] -> [n0 x][N y][N z]."""
    P, n0, n = lay.world, lay.n0, lay.n
    if P == 1:
        return ylocal
    send = ylocal.reshape(P, n0, n0, n).contiguous()  # [dest q][x_q][y_mine][z]
    recv = send.new_empty(send.shape)  # [src p][x_mine][y_p][z]
    _all_to_all(recv, send, group)
    return recv.permute(1, 0, 2, 3).reshape(n0, n, n)


def library_axis_op(precision: str = "fp64"):
    """The local step on CUDA tensors through ifdm_fft_slab, on torch's current stream."""
    import torch

    lib = _lib.load_library()
    prec = {"fp64": _lib.FP64, "fp32": _lib.FP32, "mixed": _lib.MIXED}[precision]

    def op(t, axis: int, sign: int, n: int, planes: int, poisson: bool = False, y0: int = 0):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("ifdm_fft_slab needs a contiguous CUDA tensor")
        stream = torch.cuda.current_stream(t.device).cuda_stream
        rc = lib.ifdm_fft_slab(C.c_void_p(t.data_ptr()), n, planes, axis, prec, sign, 1 if poisson else 0, y0,
                               C.c_void_p(stream))
        if rc < 0:
            raise _lib.IfdmError(rc, "ifdm_fft_slab failed")
        return t

    return op


class SlabFFT:
    """Unnormalised 3-D c2c transforms and the Poisson solve of a slab-decomposed box."""

    def __init__(self, lay: SlabLayout, axis_op=None, group=None, precision: str = "fp64"):
        self.lay = lay
        self.group = group
        self.op = axis_op or library_axis_op(precision)

    def _axis(self, t, axis, sign, poisson=False):
        lay = self.lay
        return self.op(t, axis, sign, lay.n, lay.n0, poisson, lay.x0)

    def transform(self, local, sign: int):
        """In the slab layout: sign -1 forward, +1 backward (no 1/N^3)."""
        t = self._axis(self._axis(local, 2, sign), 1, sign)
        y = self._axis(x_to_y(t, self.lay, self.group), 0, sign)
        return y_to_x(y, self.lay, self.group)

    def poisson(self, rho_local):
        """-F^-1[F[rho] / kappa^2] (normalised inverse, zero mode removed) of a
        complex slab, in the slab layout, kappa the integer wave vector; times
        4 pi G (xmax/pi)^2 its real part is the reference's phi of the density
        rho (src/CosmoBEC_MPI.cpp:80-119)."""
        t = self._axis(self._axis(rho_local, 2, -1), 1, -1)
        y = self._axis(x_to_y(t, self.lay, self.group), 0, -1, poisson=True)
        t = y_to_x(y, self.lay, self.group)
        return self._axis(self._axis(t, 1, +1), 2, +1)
